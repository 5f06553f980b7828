// Deterministic single-precision maths shared by the CUDA kernels and the CPU mirror oracle.
//
// WGSL leaves the precision of exp/log/sin/cos/pow implementation-defined, so the reference
// renderer (shaders/gps_splat.wgsl) has no bit-exact CPU twin. This header defines ONE
// implementation of each transcendental that computes the same bits on the host (g++,
// -ffp-contract=off) and on the device (nvcc --fmad=false): every step is an IEEE-754
// correctly rounded +, -, *, /, sqrt or an explicit fused multiply-add, so the result does
// not depend on the compiler or the processor.
//
// Methods (all from published mathematics, no fitted coefficients):
//   exp  : Cody & Waite (1980) argument reduction x = k ln2 + r with a two-part ln2 applied by
//          FMA, |r| <= ln2/2, then the Taylor polynomial of e^r to degree 7 (truncation error
//          r^8/8! < 6e-9 relative), scaled by 2^k through the exponent field.
//   log  : x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s), s = (m-1)/(m+1),
//          atanh series to s^11 (|s| <= 0.1716, truncation < 2e-9 relative).
//   sin/cos : Cody & Waite reduction by pi/2 (two-part constant by FMA), quadrant select,
//          Taylor polynomials of sin to r^9 and cos to r^10 on |r| <= pi/4.
// Accuracy is within a few ulp of the correctly rounded result over the ranges the renderer
// uses (tests/test_fmath.py checks it against libm in double precision and on the GPU
// against CUDA's own expf/logf/sinf/cosf).
#pragma once
#include <stdint.h>
#include <math.h>
#include <string.h>

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
constexpr float kLog2e = 1.44269502f;
constexpr float kPio2Hi = 1.57079637f;          // nearest f32 to pi/2
constexpr float kPio2Lo = -4.37113900e-08f;     // pi/2 - kPio2Hi
constexpr float kTwoOverPi = 0.636619747f;

// 2^k as a float for k in [-126, 127].
GX_HD float pow2i(int k) { return b2f((uint32_t)(k + 127) << 23); }

GX_HD float exp(float x) {
    // one range test: NaN, overflow and the subnormal/underflow tail take the slow branch
    if (!(x >= -87.3365479f && x <= 88.7228394f)) {
        if (x != x) return x;
        if (x > 88.7228394f) return b2f(0x7F800000u);
        if (x < -103.972084f) return 0.0f;
    }
    float kf = rint_(x * kLog2e);
    float r = fma_(kf, -kLn2Hi, x);
    r = fma_(kf, -kLn2Lo, r);
    // Taylor series of e^r, Horner form, coefficients 1/n!.
    float p = 1.98412698e-4f;                // 1/5040
    p = fma_(p, r, 1.38888889e-3f);          // 1/720
    p = fma_(p, r, 8.33333377e-3f);          // 1/120
    p = fma_(p, r, 4.16666679e-2f);          // 1/24
    p = fma_(p, r, 1.66666672e-1f);          // 1/6
    p = fma_(p, r, 0.5f);
    p = fma_(p, r, 1.0f);
    p = fma_(p, r, 1.0f);
    int k = (int)kf;
    if (k >= -126 && k <= 127) return p * pow2i(k);
    if (k > 127) return (p * 2.0f) * pow2i(k - 1);
    return (p * pow2i(k + 64)) * pow2i(-64);
}

GX_HD float log(float x) {
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
    e += (int)(b >> 23) - 127;
    float m = b2f((b & 0x007FFFFFu) | 0x3F800000u);
    if (m > 1.41421354f) {
        m = m * 0.5f;
        e += 1;
    }
    float f = m - 1.0f;
    float s = div_(f, 2.0f + f);
    float z = s * s;
    // 2 atanh(s) = 2 s (1 + z/3 + z^2/5 + ... + z^5/11)
    float p = 9.09090936e-2f;                // 1/11
    p = fma_(p, z, 1.11111112e-1f);          // 1/9
    p = fma_(p, z, 1.42857149e-1f);          // 1/7
    p = fma_(p, z, 2.00000003e-1f);          // 1/5
    p = fma_(p, z, 3.33333343e-1f);          // 1/3
    p = fma_(p, z, 1.0f);
    float lm = (2.0f * s) * p;
    float ef = (float)e;
    return fma_(ef, kLn2Hi, fma_(ef, kLn2Lo, lm));
}

GX_HD float sin_poly(float r) {
    float z = r * r;
    float p = 2.75573188e-6f;                // 1/9!
    p = fma_(p, z, -1.98412701e-4f);         // -1/7!
    p = fma_(p, z, 8.33333377e-3f);          // 1/5!
    p = fma_(p, z, -1.66666672e-1f);         // -1/3!
    return fma_(p * z, r, r);
}
GX_HD float cos_poly(float r) {
    float z = r * r;
    float p = -2.75573188e-7f;               // -1/10!
    p = fma_(p, z, 2.48015876e-5f);          // 1/8!
    p = fma_(p, z, -1.38888892e-3f);         // -1/6!
    p = fma_(p, z, 4.16666679e-2f);          // 1/4!
    p = fma_(p, z, -0.5f);
    return fma_(p, z, 1.0f);
}

// sin and cos of x together; accurate for |x| < 1e4 (the renderer's angles are 2 pi U).
GX_HD void sincos(float x, float* s, float* c) {
    float kf = rint_(x * kTwoOverPi);
    float r = fma_(kf, -kPio2Hi, x);
    r = fma_(kf, -kPio2Lo, r);
    float sp = sin_poly(r), cp = cos_poly(r);
    // quadrant q: odd q swaps sin and cos; sin is negated for q = 2, 3 and cos for q = 1, 2
    uint32_t q = (uint32_t)(int)kf;
    float so = (q & 1u) ? cp : sp;
    float co = (q & 1u) ? sp : cp;
    *s = b2f(f2b(so) ^ ((q & 2u) << 30));
    *c = b2f(f2b(co) ^ (((q + 1u) & 2u) << 30));
}
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
