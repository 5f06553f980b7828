// Deterministic single-precision maths shared by the CUDA kernels and the CPU mirror oracle.
//
// WGSL leaves the precision of exp/log/sin/cos/pow implementation-defined, so the reference
// renderer (shaders/gps_splat.wgsl) has no bit-exact CPU twin. This header defines ONE
// implementation of each transcendental that computes the same bits on the host (g++,
// -ffp-contract=off) and on the device (nvcc --fmad=false): every step is an IEEE-754
// correctly rounded +, -, *, /, sqrt, an explicit fused multiply-add or a read of a constant
// table (fmath_tables.h, exact float32 literals), so the result does not depend on the
// compiler or the processor.
//
// Methods (table-driven reductions after Tang, ACM TOMS 15 (1989) and 16 (1990); no fitted
// coefficients, every polynomial is a truncated Taylor series):
//   exp  : x = (64 n + j) ln2/64 + r with a two-part ln2/64 applied by FMA, |r| <= ln2/128;
//          e^x = 2^n 2^(j/64) (1 + p(r)), 2^(j/64) from a 64-entry table (high + low part),
//          p the Taylor series of e^r - 1 to degree 4 (truncation < 4e-14).
//   log  : x = 2^e m with m in [0.75, 1.5); nearest node c_i = 1 + i/128 (97-entry table of
//          RN(1/c_i) and -log RN(1/c_i)); t = m RN(1/c_i) - 1 by one FMA, |t| < 0.0053;
//          log x = e ln2 - log RN(1/c_i) + log1p(t), log1p by Taylor to degree 4.
//   sin/cos : x = j 2pi/256 + r (two-part constant by FMA), |r| <= pi/256; angle addition with
//          (sin, cos)(2 pi j/256) from a 256-entry table (high + low parts) and Taylor
//          polynomials of sin r (to r^5) and cos r - 1 (to r^4).
// Accuracy is within a few ulp of the correctly rounded result over the ranges the renderer
// uses (tests/test_fmath.py checks it against libm in double precision). The table-reading
// functions take the table base as an argument so that hot kernels can pass copies staged in
// shared memory; the plain forms read the global copies (both hold the same values).
#pragma once
#include <stdint.h>
#include <math.h>
#include <string.h>

#include "fmath_tables.h"

#if defined(__CUDACC__)
#define GX_HD __host__ __device__ __forceinline__
#else
#define GX_HD static inline
#endif

namespace gx {

GX_HD uint32_t f2b(float x) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(x);
#else
    uint32_t u;
    memcpy(&u, &x, 4);
    return u;
#endif
}
GX_HD float b2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float x;
    memcpy(&x, &u, 4);
    return x;
#endif
}

// Explicit single-rounding fused multiply-add on both sides.
GX_HD float fma_(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}
// Correctly rounded square root (IEEE-754 on both sides).
GX_HD float sqrt_(float x) {
#if defined(__CUDA_ARCH__)
    return __fsqrt_rn(x);
#else
    return sqrtf(x);
#endif
}
// Correctly rounded division.
GX_HD float div_(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
// Round to nearest, ties to even (WGSL round()).
GX_HD float rint_(float x) {
#if defined(__CUDA_ARCH__)
    return rintf(x);
#else
    return nearbyintf(x);
#endif
}
// WGSL min/max for finite operands; a NaN operand yields the other operand (IEEE minNum).
GX_HD float fmin_(float a, float b) { return fminf(a, b); }
GX_HD float fmax_(float a, float b) { return fmaxf(a, b); }
GX_HD float clamp_(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }

// WGSL u32(f32): truncation toward zero, saturated to [0, 2^32 - 1]; NaN gives 0.
GX_HD uint32_t f2u(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}

constexpr float kLn2Hi = 0.693147182f;          // nearest f32 to ln 2
constexpr float kLn2Lo = -1.904654300e-09f;     // ln 2 - kLn2Hi

// 2^k as a float for k in [-126, 127].
GX_HD float pow2i(int k) { return b2f((uint32_t)(k + 127) << 23); }

// Global table copies: the device arrays in device code, the host arrays in host code.
GX_HD const float* tab_log() {
#if defined(__CUDA_ARCH__)
    return kLogTabD;
#else
    return kLogTabH;
#endif
}
GX_HD const float* tab_exp() {
#if defined(__CUDA_ARCH__)
    return kExpTabD;
#else
    return kExpTabH;
#endif
}
GX_HD const float* tab_sc() {
#if defined(__CUDA_ARCH__)
    return kScTabD;
#else
    return kScTabH;
#endif
}
// two consecutive floats of a table (8-byte aligned pairs)
GX_HD void ld2(const float* T, int k, float* a, float* b) {
#if defined(__CUDA_ARCH__)
    float2 v = *reinterpret_cast<const float2*>(T + 2 * k);
    *a = v.x;
    *b = v.y;
#else
    *a = T[2 * k];
    *b = T[2 * k + 1];
#endif
}
// one 16-byte table row
GX_HD void ld4(const float* T, int k, float* a, float* b, float* c, float* d) {
#if defined(__CUDA_ARCH__)
    float4 v = *reinterpret_cast<const float4*>(T + 4 * k);
    *a = v.x;
    *b = v.y;
    *c = v.z;
    *d = v.w;
#else
    *a = T[4 * k];
    *b = T[4 * k + 1];
    *c = T[4 * k + 2];
    *d = T[4 * k + 3];
#endif
}

GX_HD float exp_t(float x, const float* T) {
    // one range test: NaN, overflow and the subnormal/underflow tail take the slow branch
    if (!(x >= -87.3365479f && x <= 88.7228394f)) {
        if (x != x) return x;
        if (x > 88.7228394f) return b2f(0x7F800000u);
        if (x < -103.972084f) return 0.0f;
    }
    float kf = rint_(x * kExpK);
    float r = fma_(kf, -kExpLHi, x);
    r = fma_(kf, -kExpLLo, r);
    int k = (int)kf;
    int n = k >> 6;  // k = 64 n + j
    float th, tl;
    ld2(T, k & 63, &th, &tl);
    // e^r - 1 = r + r^2 (1/2 + r/6 + r^2/24)
    float q = fma_(r, 4.16666679e-2f, 1.66666672e-1f);  // 1/24, 1/6
    q = fma_(r, q, 0.5f);
    float p = fma_(r * r, q, r);
    float v = th + fma_(th, p, tl);
    if (n >= -126 && n <= 127) return v * pow2i(n);
    if (n > 127) return (v * 2.0f) * pow2i(n - 1);
    return (v * pow2i(n + 64)) * pow2i(-64);
}
GX_HD float exp(float x) { return exp_t(x, tab_exp()); }

GX_HD float log_t(float x, const float* T) {
    uint32_t b = f2b(x);
    int e = 0;
    if (b - 0x00800000u >= 0x7F000000u) {  // one test: zero, subnormal, negative, infinite or NaN
        if (x != x || x < 0.0f) return b2f(0x7FC00000u);
        if (x == 0.0f) return b2f(0xFF800000u);
        if (b == 0x7F800000u) return x;
        x = x * 8388608.0f;  // subnormal: scale into the normal range (exact)
        b = f2b(x);
        e = -23;
    }
    const uint32_t mb = b & 0x007FFFFFu;
    const uint32_t big = mb >= 0x00400000u ? 1u : 0u;  // mantissa >= 1.5: halve it
    e += (int)(b >> 23) - 127 + (int)big;
    const float m = b2f(mb | (big ? 0x3F000000u : 0x3F800000u));  // m in [0.75, 1.5)
    const int i = (int)rint_((m - 1.0f) * 128.0f);               // nearest node, -32..64
    float rinv, thi, tlo, pad;
    ld4(T, i + 32, &rinv, &thi, &tlo, &pad);
    const float t = fma_(m, rinv, -1.0f);
    // log1p(t) = t + t^2 (-1/2 + t/3 - t^2/4)
    float q = fma_(t, -0.25f, 3.33333343e-1f);
    q = fma_(t, q, -0.5f);
    const float p = fma_(t * t, q, t);
    const float ef = (float)e;
    return fma_(ef, kLn2Hi, thi) + (fma_(ef, kLn2Lo, tlo) + p);
}
GX_HD float log(float x) { return log_t(x, tab_log()); }
// log_t for arguments known to be positive and normal (>= 2^-126, finite): the same arithmetic
// without the special-value test, so the same result bit for bit.
GX_HD float log_t_pos(float x, const float* T) {
    const uint32_t b = f2b(x);
    const uint32_t mb = b & 0x007FFFFFu;
    const uint32_t big = mb >= 0x00400000u ? 1u : 0u;
    const int e = (int)(b >> 23) - 127 + (int)big;
    const float m = b2f(mb | (big ? 0x3F000000u : 0x3F800000u));
    const int i = (int)rint_((m - 1.0f) * 128.0f);
    float rinv, thi, tlo, pad;
    ld4(T, i + 32, &rinv, &thi, &tlo, &pad);
    const float t = fma_(m, rinv, -1.0f);
    float q = fma_(t, -0.25f, 3.33333343e-1f);
    q = fma_(t, q, -0.5f);
    const float p = fma_(t * t, q, t);
    const float ef = (float)e;
    return fma_(ef, kLn2Hi, thi) + (fma_(ef, kLn2Lo, tlo) + p);
}

// sin and cos of x together; accurate for |x| < 1e4 (the renderer's angles are 2 pi U).
GX_HD void sincos_t(float x, const float* T, float* s, float* c) {
    float kf = rint_(x * kScK);
    float r = fma_(kf, -kScPHi, x);
    r = fma_(kf, -kScPLo, r);
    float sh, ch, sl, cl;
    ld4(T, (int)kf & 255, &sh, &ch, &sl, &cl);
    float z = r * r;
    float sr = fma_(z * r, fma_(z, 8.33333377e-3f, -1.66666672e-1f), r);  // sin r: 1/120, -1/6
    float cm = z * fma_(z, 4.16666679e-2f, -0.5f);                        // cos r - 1: 1/24, -1/2
    // sin(a + r) = sin a + (sin a (cos r - 1) + cos a sin r), the table's residual folded in
    *s = sh + fma_(ch, sr, fma_(sh, cm, sl));
    *c = ch + fma_(-sh, sr, fma_(ch, cm, cl));
}
GX_HD void sincos(float x, float* s, float* c) { sincos_t(x, tab_sc(), s, c); }
GX_HD float sin(float x) { float s, c; sincos(x, &s, &c); return s; }
GX_HD float cos(float x) { float s, c; sincos(x, &s, &c); return c; }

// x^y for x > 0 as exp(y log x) (used by the sRGB OETF with y = 1/2.4).
GX_HD float pow(float x, float y) {
    if (x == 0.0f) return 0.0f;
    return gx::exp(y * gx::log(x));
}

// ---------------------------------------------------------------- shared integer hashing
// PCG hash of the reference (crates/gps-core/src/lib.rs:438-442, shaders/gps_splat.wgsl:57-61).
GX_HD uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
// Frame-varying particle seed (crates/gps-core/src/lib.rs:450-465, gps_splat.wgsl:63-68).
GX_HD uint32_t particle_seed(uint32_t splat_id, uint32_t particle_index, uint32_t frame_index) {
    uint32_t s = pcg(splat_id * 747796405u + particle_index + 1u);
    s = pcg(s ^ (frame_index * 2654435761u + 1u));
    return s == 0u ? 1u : s;
}
// U[0,1) from the top 24 bits of the advanced state (gps_splat.wgsl:73-76): exact in f32.
GX_HD float next_u(uint32_t* st) {
    *st = pcg(*st);
    return (float)(*st >> 8u) * (1.0f / 16777216.0f);
}

}  // namespace gx

// Constants of the reference shader, each the f32 rounding of the WGSL abstract-float
// expression it replaces (gps_splat.wgsl line in brackets).
namespace gxc {
constexpr float kPi = 3.14159274f;               // PI [52]
constexpr float kTwoPi = 6.28318548f;            // 2.0 * PI, exact in f32
constexpr float kDilogOne = 1.64493406f;         // DILOG_ONE [53]
constexpr float kLutFv = 31.0445595f;            // 128.0 / 4.123105625617661 [121]
constexpr float kOneMinus1e6 = 0.999998987f;     // 1.0 - 1e-6 [418, 432, 435, 567, 701]
constexpr float kFrustumLim = 5.19999981f;       // 1.3 * 4.0 [176]
constexpr float kLn254over255 = -0.00392927835f; // log(1.0 - 1.0 / 255.0) [556]
constexpr float kSpMinAlpha = 0.00392156886f;    // SP_MIN_ALPHA [733]
constexpr float kInv2p4 = 0.416666657f;          // 1.0 / 2.4 (gps_composite.wgsl:31)
constexpr float kOffscreenSigma = 5.9f;          // OFFSCREEN_SIGMA [287]
constexpr float kUMin = 5.96e-8f;                // max(u, 5.96e-8) [119, 156, 407]
constexpr uint32_t kEmpty = 0xFFFFFFFFu;
}  // namespace gxc
