// Particle-path kernels for sm_100a: geometry (once per camera), Poisson counts fused with a
// single-pass decoupled-lookback scan (per ensemble), the persistent particle kernel with one
// packed 64-bit atomicMin per particle, the splat-parallel validation path, and resolve.
//
// Arithmetic follows shaders/gps_splat.wgsl expression by expression (left-to-right, IEEE f32,
// no contraction: this file is compiled with --fmad=false) with the deterministic
// transcendentals of fmath.h, so results are bit-identical to the CPU mirror oracle.
#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

#include "devmath.cuh"

// Resident blocks per SM the particle kernel is compiled for (register budget).
#ifndef GPSB_FAST_MIN_BLOCKS
#define GPSB_FAST_MIN_BLOCKS 4  // resident blocks per SM of the PBVR fast-decision variant
#endif
#ifndef GPSB_PARTICLE_MIN_BLOCKS
#define GPSB_PARTICLE_MIN_BLOCKS 5
#endif

namespace gpsb {

typedef unsigned long long ull;

// ---------------------------------------------------------------- fast decisions (PBVR)
// Most particles of a close view are never written: in the near orbit of a 560k-splat scene at
// 1280x720, 98.6 % of them fall off screen, behind the near plane or out of the radial keep test,
// and all that matters for them is whether they count as points. pbvr_fast answers that with the
// MUFU approximations (lg2 / rsqrt / sin / cos / ex2 / rcp, flush-to-zero forms) and bounds on
// |fast value - exact f32 value|; whenever a bound straddles a threshold, or the particle may
// land on screen, it answers 2 and the caller runs the exact path (emit_pbvr) from the
// particle's own stream. Its answers are therefore the exact path's:
//   0 = not a point, 1 = a point off screen (no write), 2 = undecided (run emit_pbvr).
// Error model: every standard normal the fast path draws is within kEN of the exact path's and
// at most kRMax in size (pairs with x = -2 log u1 < kXMin are left undecided), so the camera
// coordinates' bounds are per-splat constants, written by the geometry kernel into unused lanes
// of the record (fast_bounds_of); from there on, each step adds its propagated error, 2 kU per
// rounding of either path times the magnitude rounded, and kSafe for the rounding of the bound
// arithmetic itself. The constants of the approximations are checked against the exact maths
// over every input they can get (gpsb_debug_fast_bounds); the exact maths' own errors are those
// of fmath.h (exp 2 ulp, log 4 * 2^-24 relative or 2e-7 absolute).
constexpr float kU = 6.0e-8f, kSafe = 1.01f;
constexpr float kLogAbs = 3.5e-7f, kLogRel = 3.5e-7f;  // |mlog(v) - log(v)| <= kLogAbs + kLogRel |mlog(v)|, v in [kUMin, 1)
constexpr float kSinCos = 1e-6f;                    // |msin/mcos(t) - sincos(t)|, t = RN(2 pi u), u = k 2^-24
constexpr float kXMin = 1e-3f;                      // smallest x = -2 log u1 the bounds cover
constexpr float kErMax = 2.5e-6f;                   // |r - r_exact| for x >= kXMin (r = x rsqrt(x))
constexpr float kRMax = 5.77f;                      // largest r (u1 >= kUMin)
constexpr float kEN = kErMax * (1.0f + 2.0f * kSinCos) + kRMax * (kSinCos + 2.01f * kU) + 1e-7f;  // one normal
constexpr float kExpA = 6e-7f, kExpB = 1.5e-7f;     // |mexp(a) - exp(a)| <= (kExpA + kExpB |a|) mexp(a) + kExpTiny, a <= 0
constexpr float kExpTiny = 1.5e-38f;
constexpr float kLn2 = 0.693147182f, kLog2e = 1.44269502f;

__device__ __forceinline__ float mufu(float x, int op) {
    float y;
    switch (op) {
        case 0: asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); break;
        case 1: asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); break;
        case 2: asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); break;
        case 3: asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); break;
        case 4: asm("sin.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); break;
        default: asm("cos.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); break;
    }
    return y;
}
__device__ __forceinline__ float mlog(float x) { return mufu(x, 0) * kLn2; }
__device__ __forceinline__ float mexp(float a) { return mufu(a * kLog2e, 1); }

// Per-splat bounds of the fast path's camera coordinates (written by the geometry kernel into
// r1.z = |fx| ecx, r1.w = |fy| ecy, r3.z = kSafe ecz, r3.w = |a| + 2|b| + |c|, r4.w = 2(|a| + |b|),
// r5.w = 2(|b| + |c|) for the conic (a, b, c) = (r2.w, r3.x, r3.y)). World w_j = centre_j +
// sum_k L_jk u_k (2, 4, 6 operations), p = w - camera (one more), c_i = dot3(rot_i, p) (5 more).
__device__ __forceinline__ void fast_bounds_of(const FrameConst& f, float3 g0, float k00, float k10, float k11,
                                               float k20, float k21, float k22, float a, float b, float c,
                                               float4& r1, float4& r3, float4& r4, float4& r5) {
    const float sx = fabsf(k00), sy = fabsf(k10) + fabsf(k11), sz = fabsf(k20) + fabsf(k21) + fabsf(k22);
    const float gm = kRMax + kEN;
    const float Mx = fabsf(g0.x) + fabsf(f.pos[0]) + sx * gm, My = fabsf(g0.y) + fabsf(f.pos[1]) + sy * gm,
                Mz = fabsf(g0.z) + fabsf(f.pos[2]) + sz * gm;
    const float ex = sx * kEN + F_(6.0) * kU * Mx, ey = sy * kEN + F_(10.0) * kU * My, ez = sz * kEN + F_(14.0) * kU * Mz;
    auto row = [&](const float* q) {
        const float ax = fabsf(q[0]), ay = fabsf(q[1]), az = fabsf(q[2]);
        return (ax * ex + ay * ey + az * ez + F_(10.0) * kU * (ax * (Mx + ex) + ay * (My + ey) + az * (Mz + ez))) * F_(1.02);
    };
    const float ecx = row(f.rot0), ecy = row(f.rot1), ecz = row(f.rot2);
    r1.z = fabsf(f.fx) * ecx * F_(1.02);
    r1.w = fabsf(f.fy) * ecy * F_(1.02);
    r3.z = ecz * kSafe;
    r3.w = (fabsf(a) + F_(2.0) * fabsf(b) + fabsf(c)) * F_(1.02);
    r4.w = F_(2.0) * (fabsf(a) + fabsf(b)) * F_(1.02);
    r5.w = F_(2.0) * (fabsf(b) + fabsf(c)) * F_(1.02);
    if (!isfinite(ecx) || !isfinite(ecy) || !isfinite(ecz) || !isfinite(r3.w)) {
        r1.z = r1.w = r3.z = r3.w = r4.w = r5.w = __int_as_float(0x7F800000);  // never decides
    }
}

// ============================================================================ geometry
// Once per camera: projection, opacity clamp, per-method count descriptor and particle record,
// and the view-dependent SH colour (prepare/prepare_gps/prepare_pbvr without the seed-dependent
// Poisson draw, gps_splat.wgsl:535-642; splat_colour :210-251).
__global__ void __launch_bounds__(128) k_geometry(FrameConst f, const float4* __restrict__ splats,
                                                   const float* __restrict__ sh, float4* __restrict__ rec,
                                                   uint2* __restrict__ cdesc, float4* __restrict__ colour) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= f.N) return;
    float4 g0 = __ldg(&splats[4 * (size_t)i]);
    float4 g1 = __ldg(&splats[4 * (size_t)i + 1]);
    float4 g2 = __ldg(&splats[4 * (size_t)i + 2]);
    float4 g3 = __ldg(&splats[4 * (size_t)i + 3]);
    uint2 cd = make_uint2(0u, CD_NONE);
    Proj pr = project(f, g0, g1, g2);
    float o = clamp_(g0.w, F_(0.0), F_(1.0));
    float4* R = rec + (size_t)i * kRecF4;
    if (pr.ok && o > F_(0.0)) {
        float l00 = sqrt_(fmax_(pr.a, F_(1e-30)));
        float l10 = div_(pr.b, l00);
        float l11 = sqrt_(fmax_(pr.c - l10 * l10, F_(1e-30)));
        float4 r0 = make_float4(pr.mx, pr.my, pr.depth, o);
        const uint32_t method = f.method;
        const float S = (float)f.S;
        if (method == 0u && f.fp_fixed <= 1u && !(f.fp_kappa > F_(0.0))) {
            float ex = gxc::kOffscreenSigma * sqrt_(pr.a), ey = gxc::kOffscreenSigma * sqrt_(pr.c);
            bool off = pr.mx + ex < F_(0.0) || pr.mx - ex >= (float)f.W || pr.my + ey < F_(0.0) || pr.my - ey >= (float)f.H;
            if (!off) {
                float det = pr.a * pr.c - pr.b * pr.b;
                float li2 = dilog(o);
                float en = f.density * S * F_(2.0) * gxc::kPi * sqrt_(det) * li2;
                if (en > F_(0.0)) cd = make_uint2(f2b(en), CD_POISSON_CAP);
                float fo = (F_(1.0) - sqrt_(fmax_(F_(1.0) - fmin_(o, F_(1.0)), F_(0.0)))) * F_(64.0);
                uint32_t i0 = min(f2u(fo), 63u);
                float a = fo - (float)i0;
                R[0] = r0;
                R[1] = make_float4(l00, l10, l11, a);
                R[2] = make_float4(__uint_as_float(i0), li2, F_(0.0), F_(0.0));
            }
        } else if (method == 0u) {
            // footprint-subpixel mode (render_monte_carlo, oracle.rs:240-310): footprint s per splat
            // (fixed, or adaptive from the smallest standard deviation in subpixels), the expected
            // count divided by s^2, the sampling covariance optionally shrunk by the block's blur
            // (s / spp_side)^2 / 12, and the off-screen skip only for s = 1
            float det = pr.a * pr.c - pr.b * pr.b;
            uint32_t fp = max(f.fp_fixed, 1u);
            if (f.fp_kappa > F_(0.0)) {
                float tr = pr.a + pr.c;
                float disc = sqrt_(fmax_(F_(0.25) * tr * tr - det, F_(0.0)));
                float smin = sqrt_(fmax_(F_(0.5) * tr - disc, F_(0.0))) * (float)f.side;
                float sfp = floorf(f.fp_kappa * smin);
                fp = !(smin > F_(0.0)) || !(sfp >= F_(1.0)) ? 1u : (sfp >= (float)f.fp_max ? f.fp_max : (uint32_t)sfp);
            }
            float sa = pr.a, sb = pr.b, sc = pr.c;
            if (f.fp_comp && fp > 1u) {
                float q = (float)fp / (float)f.side;
                float v = q * q / F_(12.0);
                float ta = pr.a - v, tc = pr.c - v;
                float t = ta + tc, d = ta * tc - pr.b * pr.b;
                if (d > F_(0.0) && t > F_(0.0) && F_(0.5) * t - sqrt_(fmax_(F_(0.25) * t * t - d, F_(0.0))) >= v) {
                    sa = ta;
                    sc = tc;
                }
            }
            bool off = false;
            if (fp == 1u) {
                float ex = gxc::kOffscreenSigma * sqrt_(sa), ey = gxc::kOffscreenSigma * sqrt_(sc);
                off = pr.mx + ex < F_(0.0) || pr.mx - ex >= (float)f.W || pr.my + ey < F_(0.0) || pr.my - ey >= (float)f.H;
            }
            if (!off) {
                float li2 = dilog(o);
                float en = f.density * S * F_(2.0) * gxc::kPi * sqrt_(det) * li2 / (float)(fp * fp);
                if (en > F_(0.0)) cd = make_uint2(f2b(en), CD_POISSON_CAP);
                float fo = (F_(1.0) - sqrt_(fmax_(F_(1.0) - fmin_(o, F_(1.0)), F_(0.0)))) * F_(64.0);
                uint32_t i0 = min(f2u(fo), 63u);
                float a = fo - (float)i0;
                float m00 = sqrt_(fmax_(sa, F_(1e-30)));
                float m10 = div_(sb, m00);
                float m11 = sqrt_(fmax_(sc - m10 * m10, F_(1e-30)));
                R[0] = r0;
                R[1] = make_float4(m00, m10, m11, a);
                R[2] = make_float4(__uint_as_float(i0), li2, (float)fp, F_(0.0));
            }
        } else if (method == 4u) {
            float density = fmax_(f.density, F_(1e-8));
            float amin = fmax_(F_(1.0) - gx::exp(div_(gxc::kLn254over255, density)), F_(1e-8));
            if (o > amin) {
                float radius = sqrt_(F_(2.0) * gx::log(div_(o, amin)));
                float ext_x = radius * sqrt_(pr.a), ext_y = radius * sqrt_(pr.c);
                float lo_x = clamp_(floorf(pr.mx - ext_x), F_(0.0), (float)f.W);
                float lo_y = clamp_(floorf(pr.my - ext_y), F_(0.0), (float)f.H);
                float hi_x = clamp_(ceilf(pr.mx + ext_x), F_(0.0), (float)f.W);
                float hi_y = clamp_(ceilf(pr.my + ext_y), F_(0.0), (float)f.H);
                float sz_x = fmax_(hi_x - lo_x, F_(0.0)), sz_y = fmax_(hi_y - lo_y, F_(0.0));
                uint32_t count = f2u(sz_x) * f2u(sz_y) * f.side * f.side;
                if (count != 0u) {
                    float invdet = div_(F_(1.0), fmax_(pr.a * pr.c - pr.b * pr.b, F_(1e-30)));
                    float peak_tau = -gx::log(F_(1.0) - fmin_(o, gxc::kOneMinus1e6));
                    bool sparse = density * peak_tau < F_(1.0);
                    if (sparse) cd = make_uint2(f2b((float)count * density * peak_tau), CD_POISSON);
                    else cd = make_uint2(count, CD_FIXED);
                    R[0] = r0;
                    R[1] = make_float4(lo_x, lo_y, sz_x, sz_y);
                    R[2] = make_float4(pr.c * invdet, -pr.b * invdet, pr.a * invdet, peak_tau);
                    R[3] = make_float4(F_(0.0), F_(0.0), F_(0.0), sparse ? F_(1.0) : F_(0.0));
                }
            }
        } else {
            // pbvr_lambda (gps_splat.wgsl:441-460)
            float g = extinction_term(o);
            if (method == 1u) g = fmin_(o, gxc::kOneMinus1e6);
            float scale = f.base_k;
            if (method != 3u) {
                uint32_t level = f.calibration;
                if (level == 1u) scale = scale * pixel_density_scale(f, f.object_depth);
                else if (level == 2u) scale = scale * pixel_density_scale(f, pr.depth);
                else if (level == 3u) scale = S * F_(2.0) * gxc::kPi * sqrt_(pr.a * pr.c - pr.b * pr.b);
            }
            float lambda = f.density * g * scale;
            if (!(lambda > F_(0.0)) || lambda > F_(3.0e38)) lambda = F_(0.0);
            if (lambda > F_(0.0)) {
                float det = pr.a * pr.c - pr.b * pr.b;
                float keep = F_(1.0);
                uint32_t flags = CD_POISSON_CAP;
                if (method == 3u) {
                    float target = f.density * S * F_(2.0) * gxc::kPi * sqrt_(det) * dilog(o);
                    if (lambda > F_(0.5)) keep = clamp_(div_(target, lambda), F_(0.0), F_(1.0)); else keep = F_(0.0);
                    if (target > lambda) flags |= CD_UNDERCOVERED;
                }
                cd = make_uint2(f2b(lambda), flags);
                float idet = div_(F_(1.0), fmax_(det, F_(1e-30)));
                // chol_of (gps_splat.wgsl:464-485)
                float c0[3], c1[3], c2[3];
                rot_cols(g2, c0, c1, c2);
                float s2x = gx::exp(F_(2.0) * g1.x), s2y = gx::exp(F_(2.0) * g1.y), s2z = gx::exp(F_(2.0) * g1.z);
                float a00 = s2x * c0[0] * c0[0] + s2y * c1[0] * c1[0] + s2z * c2[0] * c2[0];
                float a10 = s2x * c0[1] * c0[0] + s2y * c1[1] * c1[0] + s2z * c2[1] * c2[0];
                float a20 = s2x * c0[2] * c0[0] + s2y * c1[2] * c1[0] + s2z * c2[2] * c2[0];
                float a11 = s2x * c0[1] * c0[1] + s2y * c1[1] * c1[1] + s2z * c2[1] * c2[1];
                float a21 = s2x * c0[2] * c0[1] + s2y * c1[2] * c1[1] + s2z * c2[2] * c2[1];
                float a22 = s2x * c0[2] * c0[2] + s2y * c1[2] * c1[2] + s2z * c2[2] * c2[2];
                float k00 = sqrt_(fmax_(a00, F_(1e-30)));
                float k10 = div_(a10, k00);
                float k20 = div_(a20, k00);
                float k11 = sqrt_(fmax_(a11 - k10 * k10, F_(1e-30)));
                float k21 = div_(a21 - k20 * k10, k11);
                float k22 = sqrt_(fmax_(a22 - k20 * k20 - k21 * k21, F_(1e-30)));
                float4 q1 = make_float4(keep, eol(fmin_(o, gxc::kOneMinus1e6)), F_(0.0), F_(0.0));
                float4 q3 = make_float4(-pr.b * idet, pr.a * idet, F_(0.0), F_(0.0));
                float4 q4 = make_float4(k00, k10, k11, F_(0.0));
                float4 q5 = make_float4(k20, k21, k22, F_(0.0));
                fast_bounds_of(f, make_float3(g0.x, g0.y, g0.z), k00, k10, k11, k20, k21, k22, pr.c * idet, q3.x, q3.y,
                               q1, q3, q4, q5);
                R[0] = r0;
                R[1] = q1;
                R[2] = make_float4(g0.x, g0.y, g0.z, pr.c * idet);
                R[3] = q3;
                R[4] = q4;
                R[5] = q5;
            }
        }
    }
    cdesc[i] = cd;
    if ((cd.y & 3u) != CD_NONE) colour[i] = splat_colour(f, sh, i, g0, g3);
}

void launch_geometry(const FrameConst& fc, const float4* splats, const float* sh, const float* lut, float4* rec,
                     uint2* cdesc, float4* colour, cudaStream_t st) {
    (void)lut;
    if (fc.N == 0) return;
    k_geometry<<<(fc.N + 127) / 128, 128, 0, st>>>(fc, splats, sh, rec, cdesc, colour);
}

// ============================================================================ count + scan
__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t sat_add(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    return s > kLbSumSat ? kLbSumSat : s;
}
__device__ __forceinline__ uint64_t lb_pack(uint64_t status, uint64_t sum, uint32_t nz) {
    return status | ((sum > kLbSumSat ? kLbSumSat : sum) << 24) | (uint64_t)nz;
}

// Per ensemble e and tile t of kScanTile splats: Poisson count of every splat with the stream
// particle_seed(i, 0, first_seed + e) (gps_splat.wgsl:539-548, 593-602, 573-574), the per-splat cap,
// the statistics of prepare, then a block scan and a decoupled lookback over the tiles of the
// ensemble. Splats with a non-zero count are written, in splat order, to the compact list
// clist[e * N + j] = (splat id, exclusive particle offset). The last tile writes the ensemble
// total; a total above 2^32 - 1 marks the ensemble skipped (gps_splat.wgsl:635-639, 648-654).
__global__ void __launch_bounds__(kScanThreads) k_count_scan(FrameConst f, const uint2* __restrict__ cdesc,
                                                             uint32_t first_seed, uint32_t tiles_per_e,
                                                             uint64_t* lookback, uint32_t* tile_counter,
                                                             uint2* __restrict__ clist, EnsTotal* etot, ull* stats,
                                                             uint32_t* err) {
    __shared__ uint32_t s_tile;
    __shared__ uint64_t s_wsum[kScanThreads / 32];
    __shared__ uint32_t s_wnz[kScanThreads / 32];
    __shared__ uint64_t s_excl_sum;
    __shared__ uint32_t s_excl_nz;
    __shared__ ull s_stat[6];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    if (tid < 6) s_stat[tid] = 0ull;
    __syncthreads();
    const uint32_t id = s_tile;
    const uint32_t e = id / tiles_per_e, t = id % tiles_per_e;
    const uint32_t seed = first_seed + e;
    const uint32_t N = f.N, cap = f.cap;
    const bool gps = f.method == 0u;
    const uint32_t base = t * kScanTile + tid * kScanItems;

    uint32_t cnt[kScanItems];
    ull st_pts = 0, st_trunc = 0, st_drop = 0, st_vis = 0, st_cand = 0, st_under = 0;
    uint64_t tsum = 0;
    uint32_t tnz = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        uint32_t i = base + q;
        uint32_t n = 0;
        if (i < N) {
            uint2 cd = __ldg(&cdesc[i]);
            uint32_t mode = cd.y & 3u;
            if (mode == CD_FIXED) {
                n = cd.x;
                st_cand += n;
                st_vis += 1;
            } else if (mode != CD_NONE) {
                uint32_t rs = gx::particle_seed(i, 0u, seed);
                n = poisson(__uint_as_float(cd.x), &rs);
                if (gps) st_pts += n; else st_cand += n;
                st_vis += 1;
                if (mode == CD_POISSON_CAP && n > cap) {
                    st_trunc += 1;
                    st_drop += n - cap;
                    n = cap;
                }
            }
            if (cd.y & CD_UNDERCOVERED) st_under += 1;
        }
        cnt[q] = n;
        tsum += n;
        tnz += n ? 1u : 0u;
    }
    // statistics: warp reduce, then shared, then one atomic per non-zero word per block
    ull sv[6] = {st_pts, st_trunc, st_drop, st_vis, st_cand, st_under};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        ull v = sv[k];
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(&s_stat[k], v);
    }
    // block scan of (tsum, tnz)
    uint64_t isum = tsum;
    uint32_t inz = tnz;
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t a = __shfl_up_sync(0xffffffffu, isum, o);
        uint32_t b = __shfl_up_sync(0xffffffffu, inz, o);
        if (lane >= o) { isum += a; inz += b; }
    }
    if (lane == 31) { s_wsum[warp] = isum; s_wnz[warp] = inz; }
    __syncthreads();
    uint64_t wpre = 0;
    uint32_t wpre_nz = 0, agg_nz = 0;
    uint64_t agg = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) {
        if (w < warp) { wpre += s_wsum[w]; wpre_nz += s_wnz[w]; }
        agg += s_wsum[w];
        agg_nz += s_wnz[w];
    }
    // decoupled lookback over the tiles of ensemble e
    uint64_t* lb = lookback + (size_t)e * tiles_per_e;
    if (warp == 0) {
        uint64_t excl = 0;
        uint32_t excl_nz = 0;
        if (t == 0) {
            if (lane == 0) st_relaxed(&lb[0], lb_pack(kLbPrefix, agg, agg_nz));
        } else {
            if (lane == 0) st_relaxed(&lb[t], lb_pack(kLbAggregate, agg, agg_nz));
            int32_t pred = (int32_t)t - 1;
            uint32_t spins = 0;
            bool failed = false;
            while (true) {
                int32_t j = pred - lane;
                uint64_t w = 0;
                if (j >= 0) {
                    w = ld_relaxed(&lb[j]);
                    while ((w >> 62) == 0ull) {
                        if (++spins > (1u << 20)) { failed = true; break; }
                        __nanosleep(64);
                        w = ld_relaxed(&lb[j]);
                    }
                } else {
                    w = kLbPrefix;  // before tile 0: an empty inclusive prefix
                }
                if (__any_sync(0xffffffffu, failed)) { failed = true; break; }
                uint32_t is_prefix = __ballot_sync(0xffffffffu, (w >> 62) == 2ull);
                int first = is_prefix ? __ffs(is_prefix) - 1 : 32;  // closest predecessor with a prefix
                uint64_t v_sum = (lane <= first) ? ((w >> 24) & kLbSumSat) : 0ull;
                uint32_t v_nz = (lane <= first) ? (uint32_t)(w & 0xFFFFFFull) : 0u;
                for (int o = 16; o; o >>= 1) {
                    v_sum += __shfl_xor_sync(0xffffffffu, v_sum, o);
                    v_nz += __shfl_xor_sync(0xffffffffu, v_nz, o);
                }
                excl = sat_add(excl, v_sum);
                excl_nz += v_nz;
                if (first < 32) break;
                pred -= 32;
            }
            if (failed) {
                if (lane == 0) {
                    atomicOr(err, ERR_SCAN_LOOKBACK);
                    atomicOr(&etot[e].flags, 2u);
                }
                excl = 0;
                excl_nz = 0;
            }
            if (lane == 0) st_relaxed(&lb[t], lb_pack(kLbPrefix, sat_add(excl, agg), excl_nz + agg_nz));
        }
        if (lane == 0) { s_excl_sum = excl; s_excl_nz = excl_nz; }
    }
    __syncthreads();
    // compact list of non-zero splats
    uint64_t off = s_excl_sum + wpre + (isum - tsum);
    uint32_t j = s_excl_nz + wpre_nz + (inz - tnz);
    uint2* out = clist + (size_t)e * N;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        if (cnt[q]) {
            out[j] = make_uint2(base + q, (uint32_t)off);
            off += cnt[q];
            ++j;
        }
    }
    if (tid < 6 && s_stat[tid]) {
        const int word[6] = {ST_POINTS, ST_TRUNCATED, ST_DROPPED, ST_VISIBLE, ST_CANDIDATES, ST_UNDERCOVERED};
        atomicAdd(&stats[word[tid]], s_stat[tid]);
    }
    if (t == tiles_per_e - 1 && tid == 0) {
        uint64_t total = sat_add(s_excl_sum, agg);
        etot[e].particles = total;
        etot[e].nonzero = s_excl_nz + agg_nz;
        atomicAdd(&stats[ST_ENTRIES], (ull)(s_excl_nz + agg_nz));
        if (total > 0xFFFFFFFFull) {
            atomicOr(&etot[e].flags, 1u);
            atomicAdd(&stats[ST_SKIPPED], 1ull);
        } else {
            atomicAdd(&stats[ST_PARTICLES], (ull)total);
        }
    }
}

void launch_count_scan(const FrameConst& fc, const uint2* cdesc, uint32_t first_seed, uint32_t E, uint64_t* lookback,
                       uint32_t* tile_counter, uint2* clist, EnsTotal* etot, unsigned long long* stats, uint32_t* err,
                       cudaStream_t st) {
    uint32_t tiles = (fc.N + kScanTile - 1) / kScanTile;
    cudaMemsetAsync(lookback, 0, (size_t)E * tiles * sizeof(uint64_t), st);
    cudaMemsetAsync(tile_counter, 0, sizeof(uint32_t), st);
    cudaMemsetAsync(etot, 0, (size_t)E * sizeof(EnsTotal), st);
    if (fc.N == 0 || E == 0) return;
    k_count_scan<<<tiles * E, kScanThreads, 0, st>>>(fc, cdesc, first_seed, tiles, lookback, tile_counter, clist, etot,
                                                      stats, err);
}

// ============================================================================ particles
constexpr int kLutN = 65 * 129;

__device__ __forceinline__ void splat_write(ull* sub, uint32_t idx, float depth_z, uint32_t id) {
    ull packed = ((ull)(f2b(depth_z) | 0x80000000u) << 32) | (ull)id;
    ull cur = __ldcg(sub + idx);
    if (packed < cur) atomicMin(sub + idx, packed);
}

// emit_particle (gps_splat.wgsl:259-282) with the packed winner rule
__device__ __forceinline__ uint32_t emit_gps(const FrameConst& f, const FTabs& T, const float* lut, uint32_t i, uint32_t& rs,
                                             float4 r0, float4 r1, float4 r2, ull* sub) {
    float u = gx::next_u(&rs);
    float r = f.exact_radius ? corrected_radius_exact(r0.w, r2.y, u)
                             : corrected_radius_lut(lut, __float_as_uint(r2.x), r1.w, u, T.lg);
    float th = gxc::kTwoPi * gx::next_u(&rs);
    float sn, cs;
    gx::sincos_t(th, T.sc, &sn, &cs);
    float wx = r * cs, wy = r * sn;
    float px_ = r0.x + r1.x * wx;
    float py_ = r0.y + (r1.y * wx + r1.z * wy);
    if (r2.z > F_(1.0)) {
        // footprint block (write_block, oracle.rs:156-173): the s x s subpixels around the sample
        const int s = (int)r2.z, side = (int)f.side;
        const int gx0 = (int)floorf(px_ * (float)side - F_(0.5) * (float)s + F_(0.5));
        const int gy0 = (int)floorf(py_ * (float)side - F_(0.5) * (float)s + F_(0.5));
        const int gw = (int)f.W * side, gh = (int)f.H * side;
        uint32_t wrote = 0u;
        for (int gy = max(gy0, 0); gy < min(gy0 + s, gh); ++gy)
            for (int gx = max(gx0, 0); gx < min(gx0 + s, gw); ++gx) {
                const uint32_t qx = (uint32_t)(gx / side), qy = (uint32_t)(gy / side);
                splat_write(sub, (qy * f.W + qx) * f.S + (uint32_t)(gy % side) * f.side + (uint32_t)(gx % side), r0.z, i);
                wrote = 1u;
            }
        return wrote;
    }
    if (px_ < F_(0.0) || px_ >= (float)f.W || py_ < F_(0.0) || py_ >= (float)f.H) return 0u;
    uint32_t px = f2u(px_), py = f2u(py_);
    uint32_t sx = min(f.side - 1u, f2u((px_ - (float)px) * (float)f.side));
    uint32_t sy = min(f.side - 1u, f2u((py_ - (float)py) * (float)f.side));
    splat_write(sub, (py * f.W + px) * f.S + sy * f.side + sx, r0.z, i);
    return 1u;
}

struct Normal {
    uint32_t* st;
    const FTabs& T;
    bool has;
    float spare;
    __device__ __forceinline__ float next() {
        if (has) { has = false; return spare; }
        float u1 = fmax_(gx::next_u(st), gxc::kUMin);
        float u2 = gx::next_u(st);
        float r = sqrt_(-F_(2.0) * gx::log_t_pos(u1, T.lg));  // u1 >= kUMin
        float sn, cs;
        gx::sincos_t(gxc::kTwoPi * u2, T.sc, &sn, &cs);
        spare = r * sn;
        has = true;
        return r * cs;
    }
};

// emit_particle_pbvr (gps_splat.wgsl:490-532); returns bit 0 = counts as a point, bit 1 = written
__device__ __forceinline__ uint32_t emit_pbvr(const FrameConst& f, const FTabs& T, uint32_t i, uint32_t& rs, const float4* R,
                                              ull* sub) {
    Normal nm{&rs, T, false, F_(0.0)};
    float uz = nm.next();
    float uy = nm.next();
    float ux = nm.next();
    float4 r1 = R[1];
    if (f.method == 3u) {
        if (gx::next_u(&rs) >= r1.x) return 0u;
    }
    float4 r2 = R[2], r4 = R[4], r5 = R[5];
    float wx = r2.x + r4.x * ux;
    float wy = r2.y + (r4.y * ux + r4.z * uy);
    float wz = r2.z + (r5.x * ux + r5.y * uy + r5.z * uz);
    float px = wx - f.pos[0], py = wy - f.pos[1], pz = wz - f.pos[2];
    float cx = dot3(f.rot0[0], f.rot0[1], f.rot0[2], px, py, pz);
    float cy = dot3(f.rot1[0], f.rot1[1], f.rot1[2], px, py, pz);
    float cz = dot3(f.rot2[0], f.rot2[1], f.rot2[2], px, py, pz);
    if (cz <= f.near_z) return 0u;
    float pix_x = div_(f.fx * cx, cz) + f.cx;
    float pix_y = div_(f.fy * cy, cz) + f.cy;
    const uint32_t flags = f.flags;
    if (flags & FLAG_JITTER) {
        float jy = nm.next();
        float jx = nm.next();
        pix_x = pix_x + f.jitter_sd * jx;
        pix_y = pix_y + f.jitter_sd * jy;
    }
    float4 r0 = R[0];
    if (flags & FLAG_RADIAL) {
        float4 r3 = R[3];
        float dvx = pix_x - r0.x, dvy = pix_y - r0.y;
        float r2v = r2.w * dvx * dvx + F_(2.0) * r3.x * dvx * dvy + r3.y * dvy * dvy;
        // radial_keep (gps_splat.wgsl:434-438) with h(min(o, 1-1e-6)) hoisted per splat
        float oo = fmin_(r0.w, gxc::kOneMinus1e6);
        float y = oo * gx::exp_t(-F_(0.5) * fmax_(r2v, F_(0.0)), T.ex);
        float keep = clamp_(div_(eol(y, T.lg), r1.y), F_(0.0), F_(1.0));
        if (gx::next_u(&rs) >= keep) return 0u;
    }
    float depth_z = (flags & FLAG_CENTRE) ? r0.z : cz;
    if (pix_x < F_(0.0) || pix_x >= (float)f.W || pix_y < F_(0.0) || pix_y >= (float)f.H) return 1u;
    uint32_t ipx = f2u(pix_x), ipy = f2u(pix_y);
    uint32_t sx = min(f.side - 1u, f2u((pix_x - (float)ipx) * (float)f.side));
    uint32_t sy = min(f.side - 1u, f2u((pix_y - (float)ipy) * (float)f.side));
    splat_write(sub, (ipy * f.W + ipx) * f.S + sy * f.side + sx, depth_z, i);
    return 3u;
}

// One Box-Muller pair from the stream, drawn in the order of Normal::next (cos part, sin part).
// Returns false when x = -2 log u1 is below kXMin, where the kEN bound does not hold.
__device__ __forceinline__ bool fast_pair(uint32_t& st, float& c, float& s) {
    const float u1 = fmax_(gx::next_u(&st), gxc::kUMin);
    st = gx::pcg(st);  // u2 = (st >> 8) 2^-24, folded into t below
    // x = -2 mlog(u1) and t = RN(2 pi u2), each with one rounding: scaling by a power of two
    // commutes with rounding, so both equal the two-step values bit for bit
    const float x = mufu(u1, 0) * (-F_(2.0) * kLn2);
    const float r = x * mufu(x, 2);
    const float t = (float)(st >> 8u) * (gxc::kTwoPi * (F_(1.0) / F_(16777216.0)));
    c = r * mufu(t, 5);
    s = r * mufu(t, 4);
    return x >= kXMin;
}

// Straight-line form: every lane computes the whole path and the answer is selected at the end
// (the lanes of a warp rarely agree on an early exit, and divergent exits cost more than they save).
__device__ __forceinline__ uint32_t pbvr_fast(const FrameConst& f, uint32_t st, const float4* R) {
    float uz, uy, ux, jy;
    bool ok = fast_pair(st, uz, uy);
    ok &= fast_pair(st, ux, jy);  // jy is the pair's spare, used by the jitter
    const float4 r1 = R[1];
    if (f.method == 3u) {
        if (gx::next_u(&st) >= r1.x) return 0u;  // the exact draw and test
    }
    const float4 r2 = R[2], r3 = R[3], r4 = R[4], r5 = R[5];
    const float px = __fmaf_rn(r4.x, ux, r2.x) - f.pos[0];
    const float py = __fmaf_rn(r4.z, uy, __fmaf_rn(r4.y, ux, r2.y)) - f.pos[1];
    const float pz = __fmaf_rn(r5.z, uz, __fmaf_rn(r5.y, uy, __fmaf_rn(r5.x, ux, r2.z))) - f.pos[2];
    const float cz = __fmaf_rn(f.rot2[2], pz, __fmaf_rn(f.rot2[1], py, f.rot2[0] * px));
    const float ecz = r3.z;  // already widened by kSafe
    const bool behind = cz + ecz <= f.near_z;  // surely not a point
    const float czl = cz - ecz;
    bool sure = czl > f.near_z && czl > F_(3.0) * ecz && cz < 1e30f && czl > 1e-6f;  // surely in front
    const float cx = __fmaf_rn(f.rot0[2], pz, __fmaf_rn(f.rot0[1], py, f.rot0[0] * px));
    const float cy = __fmaf_rn(f.rot1[2], pz, __fmaf_rn(f.rot1[1], py, f.rot1[0] * px));
    // t = (f c) / cz; |t - t'| <= (|f| ec + |t| ecz) / (cz - ecz) + the reciprocal's and both
    // paths' roundings (1e-6 |t|), 1 / (cz - ecz) <= (1 + 2 ecz / cz) / cz for ecz <= cz / 4;
    // then + f.cx with one more rounding in each path
    const float icz = mufu(cz, 3);
    const float icl = icz * __fmaf_rn((F_(2.0) * kSafe) * ecz, icz, kSafe);
    const float kt = __fmaf_rn(ecz, icl, 1e-6f + F_(2.0) * kU);
    const float tx = (f.fx * cx) * icz, ty = (f.fy * cy) * icz;
    float pix_x = tx + f.cx, pix_y = ty + f.cy;
    float epx = __fmaf_rn(fabsf(tx), kt, __fmaf_rn(r1.z, icl, F_(2.0) * kU * fabsf(f.cx)));
    float epy = __fmaf_rn(fabsf(ty), kt, __fmaf_rn(r1.w, icl, F_(2.0) * kU * fabsf(f.cy)));
    const uint32_t flags = f.flags;
    if (flags & FLAG_JITTER) {
        float jx, js;
        sure &= fast_pair(st, jx, js);
        // |sd j - sd j'| <= |sd| kEN, + the product's and the sum's roundings in both paths
        const float kj = fabsf(f.jitter_sd) * (kEN + F_(4.0) * kU * kRMax);
        pix_x = pix_x + f.jitter_sd * jx;
        pix_y = pix_y + f.jitter_sd * jy;
        epx = __fmaf_rn(F_(4.0) * kU, fabsf(pix_x), epx + kj);
        epy = __fmaf_rn(F_(4.0) * kU, fabsf(pix_y), epy + kj);
    }
    sure &= fabsf(pix_x) < 1e30f && fabsf(pix_y) < 1e30f && epx < 1e30f && epy < 1e30f;
    const float mx = kSafe * epx, my = kSafe * epy;
    const bool off = pix_x + mx < F_(0.0) || pix_x - mx >= (float)f.W || pix_y + my < F_(0.0) || pix_y - my >= (float)f.H;
    uint32_t res = off ? 1u : 2u;
    if (flags & FLAG_RADIAL) {
        const float4 r0 = R[0];
        const float dvx = pix_x - r0.x, dvy = pix_y - r0.y;
        const float e = fmaxf(__fmaf_rn(F_(2.0) * kU, fabsf(pix_x) + fabsf(r0.x), epx),
                              __fmaf_rn(F_(2.0) * kU, fabsf(pix_y) + fabsf(r0.y), epy));
        // r2v = a dx^2 + 2 b dx dy + c dy^2: |grad . d| <= e (G_x |dx| + G_y |dy|), |Q(d)| <= K e^2,
        // roundings <= 20 kU (|a| + |b|) dx^2 + (|b| + |c|) dy^2
        const float dx2 = dvx * dvx, dy2 = dvy * dvy;
        const float r2v = __fmaf_rn(r2.w, dx2, __fmaf_rn(F_(2.0) * r3.x, dvx * dvy, r3.y * dy2));
        const float m2 = __fmaf_rn(r4.w, dx2, r5.w * dy2);
        const float er2 = __fmaf_rn(__fmaf_rn(r4.w, fabsf(dvx), r5.w * fabsf(dvy)), e, __fmaf_rn(r3.w * e, e, F_(10.0) * kU * m2));
        const float a2 = fmaxf(r2v, F_(0.0));  // arg = -a2 / 2
        const float earg = er2 * (F_(0.5) * kSafe);
        // y = min(o, 1 - 1e-6) exp(arg): propagated error (e^earg - 1 <= earg (1 + earg)), the
        // approximation against exp, exp's own 2 ulp at both arguments, the product's roundings;
        // with earg < 1/8 every relative term grows by at most (1 + 2 earg) <= 1.25
        const float oo = fmin_(r0.w, gxc::kOneMinus1e6);
        const float y = oo * mufu(a2 * (-F_(0.5) * kLog2e), 1);  // = mexp(arg) bit for bit
        const float rel = __fmaf_rn(earg, F_(1.0) + earg, __fmaf_rn(F_(0.5) * kExpB, a2, kExpA + F_(5.4e-7) + F_(2.0) * kU));
        const float ey = __fmaf_rn(y, rel * (F_(1.25) * kSafe), F_(2.02) * kExpTiny);
        // eol's log form, eol(y) = -log(1 - y) / y, which both paths take when y - ey >= 1e-4 (the
        // short form 1 + y / 2 of y < 1e-4, beyond ~4.3 standard deviations, is left to the exact
        // path), with 1 / (a - e) <= (1 + 2 e / a) / a for e <= a / 2: the approximation against
        // log at v, log's own error at both arguments, the argument's error
        const float v = F_(1.0) - fmin_(y, gxc::kOneMinus1e6);
        const float ev = ey + F_(2.0) * kU;
        const float lg = mlog(v);
        const float iv = mufu(v, 3), iy = mufu(y, 3);
        const float elg = __fmaf_rn(kLogRel + F_(5e-7), fabsf(lg), kLogAbs + F_(4e-7)) +
                          ev * iv * __fmaf_rn(F_(2.0) * ev, iv, F_(1.0)) * kSafe;
        const float eo = -lg * iy;
        const float eeo = __fmaf_rn(__fmaf_rn(fabsf(eo), ey, elg) * iy, __fmaf_rn(F_(2.0) * ey, iy, F_(1.0)) * kSafe,
                                    F_(4e-7) * fabsf(eo));
        sure &= earg < F_(0.125) && y - ey >= F_(1e-4) && ev <= F_(0.5) * v && ey <= F_(0.5) * y;
        const float de = eeo * kSafe;
        // keep = clamp(eo / r1.y, 0, 1) against the exact draw, compared as u r1.y against eo
        const float ur = gx::next_u(&st) * r1.y;
        const bool reject = ur >= (eo + de) * (F_(1.0) + F_(6.0) * kU);
        const bool keep = ur * (F_(1.0) + F_(6.0) * kU) < eo - de;
        res = reject ? 0u : (keep ? res : 2u);
    }
    res = behind ? 0u : (sure ? res : 2u);
    return ok ? res : 2u;
}

// Exhaustive check of the constants of the fast decisions: the largest |approximation - exact| /
// bound over every input the approximations get, out[0..5] as float bits (ratios <= 1 hold the
// bounds): log over the uniforms k 2^-24; log over every float in [1e-6, 1); sin and cos over
// 2 pi k 2^-24; |r - r_exact| / kErMax over the uniforms with x >= kXMin; r / kRMax; exp over
// every float in [-128, 0]. NaN shows as infinity.
__device__ __forceinline__ void upd_ratio(float& m, float v) { m = v != v ? __int_as_float(0x7F800000) : fmaxf(m, v); }

__global__ void __launch_bounds__(256) k_fast_bounds(uint32_t* out) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    float m[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (uint32_t k = tid; k < (1u << 24); k += nth) {
        const float u = (float)k * (1.0f / 16777216.0f);
        const float u1 = fmax_(u, gxc::kUMin);
        const float L = mlog(u1), Le = gx::log(u1);
        upd_ratio(m[0], fabsf(L - Le) / __fmaf_rn(kLogRel, fabsf(L), kLogAbs));
        // r exactly as fast_pair and Normal::next compute it
        const float x = -F_(2.0) * L;
        const float r = x * mufu(x, 2);
        const float re = sqrt_(-F_(2.0) * Le);
        if (x >= kXMin) {
            upd_ratio(m[3], fabsf(r - re) / kErMax);
            upd_ratio(m[4], r / kRMax);
        }
        const float t = gxc::kTwoPi * u;
        float se, ce;
        gx::sincos(t, &se, &ce);
        upd_ratio(m[2], fmaxf(fabsf(mufu(t, 4) - se), fabsf(mufu(t, 5) - ce)) / kSinCos);
    }
    for (uint32_t b = __float_as_uint(1e-6f) + tid; b < 0x3F800000u; b += nth) {
        const float v = __uint_as_float(b);
        const float L = mlog(v);
        upd_ratio(m[1], fabsf(L - gx::log(v)) / __fmaf_rn(kLogRel, fabsf(L), kLogAbs));
    }
    for (uint32_t b = 0x80000000u + tid; b <= 0xC3000000u; b += nth) {
        const float a = __uint_as_float(b);
        const float y = mexp(a);
        upd_ratio(m[5], fabsf(y - gx::exp(a)) / __fmaf_rn(__fmaf_rn(kExpB, fabsf(a), kExpA), y, kExpTiny));
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        const uint32_t w = __reduce_max_sync(0xffffffffu, __float_as_uint(m[c]));
        if ((threadIdx.x & 31) == 0 && w) atomicMax(&out[c], w);
    }
}

void launch_fast_bounds(uint32_t* out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, 6 * sizeof(uint32_t), st);
    k_fast_bounds<<<148 * 8, 256, 0, st>>>(out);
}

// ScreenOccupancy branch of particle_pass (gps_splat.wgsl:686-708); returns 1 on a hit
__device__ __forceinline__ uint32_t emit_so(const FrameConst& f, const FTabs& T, uint32_t i, uint32_t k, uint32_t& rs,
                                            const float4* R, ull* sub) {
    float4 r0 = R[0], b = R[1];
    const uint32_t side = f.side, samples = f.S;
    bool sparse = R[3].w > F_(0.0);
    uint32_t cell = k;
    uint32_t bz = f2u(b.z), bw = f2u(b.w);
    if (sparse) cell = min(f2u(gx::next_u(&rs) * b.z * b.w * (float)samples), bz * bw * samples - 1u);
    uint32_t pixel = cell / samples, sub_i = cell % samples;
    uint32_t xx = f2u(b.x) + pixel % bz, yy = f2u(b.y) + pixel / bz;
    float n1 = gx::next_u(&rs);
    float n2 = gx::next_u(&rs);
    float uvx = div_((float)(sub_i % side) + n1, (float)side);
    float uvy = div_((float)(sub_i / side) + n2, (float)side);
    float dx = (float)xx + uvx - r0.x, dy = (float)yy + uvy - r0.y;
    float4 inv = R[2];
    float r2 = fmax_(inv.x * dx * dx + F_(2.0) * inv.y * dx * dy + inv.z * dy * dy, F_(0.0));
    float alpha = fmin_(r0.w * gx::exp_t(-F_(0.5) * r2, T.ex), gxc::kOneMinus1e6);
    float coverage;
    if (sparse) coverage = div_(-gx::log_t(F_(1.0) - alpha, T.lg), inv.w);
    else coverage = F_(1.0) - gx::exp_t(f.density * gx::log_t(F_(1.0) - alpha, T.lg), T.ex);
    if (gx::next_u(&rs) >= coverage) return 0u;
    splat_write(sub, (yy * f.W + xx) * samples + sub_i, r0.z, i);
    return 1u;
}

constexpr int kPT = 256;               // threads per particle block
constexpr uint32_t kRing = 64;         // per-warp ring of undecided PBVR particles (uint2 entries)
#ifndef GPSB_FAST_GIVE_UP
#define GPSB_FAST_GIVE_UP 10
#endif
// undecided lanes of one step above which a warp stops the fast test for the rest of its tile
// (measured on the bench views: 10 beats 4, 7, 16, 24 and never giving up)
constexpr uint32_t kFastGiveUp = GPSB_FAST_GIVE_UP;
static_assert(kTabFloats % 2 == 0, "the ring after the entry lists needs 8-byte alignment");

// Largest j in [lo, hi) with off(j) <= v, by a 32-ary warp search (off(lo) <= v must hold).
__device__ __forceinline__ uint32_t warp_last_le(const uint2* __restrict__ L, uint32_t lo, uint32_t hi, uint64_t v, int lane) {
    while (hi - lo > 1u) {
        uint32_t n = hi - lo;
        uint32_t step = (n + 31u) / 32u;
        uint32_t idx = lo + (uint32_t)(lane + 1) * step;
        bool p = idx < hi && (uint64_t)__ldg(&L[idx].y) <= v;
        uint32_t c = __popc(__ballot_sync(0xffffffffu, p));
        uint32_t nlo = lo + c * step;
        uint32_t nhi = lo + (c + 1u) * step;
        lo = nlo;
        hi = nhi < hi ? nhi : hi;
    }
    return lo;
}

// Persistent particle kernel: every block repeatedly takes a tile of kPTile consecutive
// particles of one ensemble (dynamic work counter), maps each particle to (splat i, k) through
// the compact list, regenerates it from its own stream particle_seed(i, k + 1, seed) and writes it
// with one 64-bit atomicMin of (depth key << 32 | i), which equals the reference's depth pass
// followed by the colour pass (gps_splat.wgsl:276-281). Ensembles flagged skipped get no work.
// MC: 0 GPS, 1 PBVR, 2 ScreenOccupancy; kPIPT: particles per thread per tile; FM: PBVR fast decisions
// (0 off, 1 on, 2 validate), a template parameter so each variant gets its own register allocation
template <int MC, int kPIPT, int FM>
__global__ void __launch_bounds__(kPT, FM == 1 ? GPSB_FAST_MIN_BLOCKS : GPSB_PARTICLE_MIN_BLOCKS) k_particles(FrameConst f, const float4* __restrict__ rec,
                                                   const float* __restrict__ lut, const uint2* __restrict__ clist,
                                                   const EnsTotal* __restrict__ etot, uint32_t first_seed, uint32_t E,
                                                   ull* sub, uint32_t* unit_counter, ull* stats) {
    constexpr int kPTile = kPT * kPIPT;  // particles per tile
    // dynamic shared memory: [fmath tables (kTabFloats)] [first unit of each ensemble (E + 1)]
    // [entry offsets (kPTile + 2)] [entry ids (kPTile + 2)] [radius table (GPS) | rings (PBVR fast)]
    extern __shared__ __align__(16) uint32_t s_dyn[];
    const FTabs T = stage_tabs(reinterpret_cast<float*>(s_dyn));
    uint64_t* s_ubase = reinterpret_cast<uint64_t*>(s_dyn + kTabFloats);
    uint32_t* s_off = s_dyn + kTabFloats + 2 * (E + 1);
    uint32_t* s_id = s_off + (kPTile + 2);
    float* s_lut = reinterpret_cast<float*>(s_id + (kPTile + 2));
    __shared__ uint32_t s_unit, s_j0, s_w, s_claim;
    const int tid = threadIdx.x, lane = tid & 31;
    const bool use_lut = MC == 0 && !f.exact_radius;
    if (use_lut)
        for (int k = tid; k < kLutN; k += kPT) s_lut[k] = __ldg(&lut[k]);
    if (tid == 0) {
        uint64_t acc = 0;
        for (uint32_t e = 0; e < E; ++e) {
            s_ubase[e] = acc;
            EnsTotal t = etot[e];
            if (t.flags == 0u && t.particles) acc += (t.particles + kPTile - 1) / kPTile;
        }
        s_ubase[E] = acc;
    }
    __syncthreads();
    const uint64_t total_units = s_ubase[E];
    const uint64_t PS = (uint64_t)f.W * f.H * f.S;
    uint32_t points = 0, writes = 0, exact_runs = 0, mismatch = 0;
    // next tile: its unit number and list window, found by one warp (lane 0 writes s_unit, s_j0, s_w)
    auto find_unit = [&]() {
        uint32_t un = 0u;
        if (lane == 0) un = atomicAdd(unit_counter, 1u);
        un = __shfl_sync(0xffffffffu, un, 0);
        uint32_t j0 = 0u, j1 = 0u;
        if ((uint64_t)un < total_units) {
            uint32_t lo = 0, hi = E;
            while (hi - lo > 1u) {
                uint32_t mid = (lo + hi) >> 1;
                if (s_ubase[mid] <= un) lo = mid; else hi = mid;
            }
            const EnsTotal et = etot[lo];
            const uint64_t q0 = ((uint64_t)un - s_ubase[lo]) * kPTile;
            const uint64_t q1 = q0 + kPTile < et.particles ? q0 + kPTile : et.particles;
            const uint2* Lq = clist + (size_t)lo * f.N;
            j0 = warp_last_le(Lq, 0u, et.nonzero, q0, lane);
            j1 = warp_last_le(Lq, j0, et.nonzero, q1 - 1, lane);
        }
        if (lane == 0) {
            s_unit = un;
            s_j0 = j0;
            s_w = j1 - j0 + 1u;
        }
    };
    if (tid < 32) find_unit();
    __syncthreads();
    for (;;) {
        const uint64_t u = s_unit;
        if (u >= total_units) break;
        const uint32_t j0 = s_j0, w = s_w;
        // ensemble of unit u: largest e with s_ubase[e] <= u
        uint32_t lo = 0, hi = E;
        while (hi - lo > 1u) {
            uint32_t mid = (lo + hi) >> 1;
            if (s_ubase[mid] <= u) lo = mid; else hi = mid;
        }
        const uint32_t e = lo;
        const EnsTotal et = etot[e];
        const uint64_t p0 = (u - s_ubase[e]) * kPTile;
        const uint64_t p1 = p0 + kPTile < et.particles ? p0 + kPTile : et.particles;
        const uint2* L = clist + (size_t)e * f.N;
        for (uint32_t q = tid; q <= w; q += kPT) {
            uint32_t j = j0 + q;
            if (q < w) {
                uint2 ent = __ldg(&L[j]);
                s_id[q] = ent.x;
                s_off[q] = ent.y;
            } else {
                s_off[q] = j < et.nonzero ? __ldg(&L[j].y) : (uint32_t)et.particles;
            }
        }
        if (tid == 0) s_claim = 0u;
        __syncthreads();  // window staged, unit read by every thread, claim open
        const uint32_t seed = first_seed + e;
        ull* S = sub + (size_t)e * PS;
        uint64_t p = p0 + (uint64_t)tid * kPIPT;
        if (MC == 1 && FM == 1) {
            // Converged warp loop over the fast decisions: the particles pbvr_fast leaves undecided
            // go to a per-warp ring in shared memory and run the exact path 32 at a time with the
            // whole warp, instead of once for every divergent lane. A warp whose lanes are mostly
            // undecided (on-screen work) drops the fast test for the rest of the tile.
            uint2* ring = reinterpret_cast<uint2*>(s_lut) + (size_t)(tid >> 5) * kRing;
            const uint32_t below = (1u << lane) - 1u;
            uint32_t head = 0u, count = 0u, pp = 0u, pend = 0u, jj = 0u, cur = 0xFFFFFFFFu;
            bool fast = true;
            float4 R[kRecF4];
            if (p < p1) {
                pp = (uint32_t)p;
                uint32_t a = 0, b = w;
                while (b - a > 1u) {
                    uint32_t m = (a + b) >> 1;
                    if (s_off[m] <= pp) a = m; else b = m;
                }
                jj = a;
                pend = (uint32_t)(p + kPIPT < p1 ? p + kPIPT : p1);
            }
            auto load_rec = [&](uint32_t i) {
                const float4* Rg = rec + (size_t)i * kRecF4;
#pragma unroll
                for (int c = 0; c < kRecF4; ++c) R[c] = __ldg(&Rg[c]);
                cur = i;
            };
            auto run_exact = [&](uint32_t i, uint32_t k) {
                if (i != cur) load_rec(i);
                uint32_t rs = gx::particle_seed(i, k + 1u, seed);
                const uint32_t r = emit_pbvr(f, T, i, rs, R, S);
                points += r & 1u;
                writes += r >> 1;
            };
            uint32_t nxt = 0u, ci = 0u, ck = 0u;  // next entry boundary, current splat and index
            if (pp < pend) {
                ci = s_id[jj];
                ck = pp - s_off[jj];
                nxt = s_off[jj + 1];
            }
            // fast steps: every lane evaluates a particle (a lane past its range evaluates one it
            // does not own and ignores the answer; pbvr_fast only reads registers), so the step
            // body has no divergent branch but the list boundary; a warp whose splat changed in
            // any lane reloads every lane's record
            int it = 0;
            for (; it < kPIPT && fast; ++it) {
                const bool act = pp < pend;
                if (act && pp >= nxt) {
                    while (pp >= s_off[jj + 1]) ++jj;
                    ci = s_id[jj];
                    ck = pp - s_off[jj];
                    nxt = s_off[jj + 1];
                }
                const uint32_t i = ci, k = ck;
                ck += act ? 1u : 0u;
                pp += act ? 1u : 0u;
                if (__any_sync(0xffffffffu, i != cur)) load_rec(i);
                const uint32_t q = pbvr_fast(f, gx::particle_seed(i, k + 1u, seed), R);
                const uint32_t need = (act && q == 2u) ? 1u : 0u;
                points += (act && q != 2u) ? q : 0u;
                const uint32_t bal = __ballot_sync(0xffffffffu, need);
                if (bal == 0u) continue;
                const uint32_t n = (uint32_t)__popc(bal);
                if (need) ring[(head + count + (uint32_t)__popc(bal & below)) & (kRing - 1u)] = make_uint2(i, k);
                count += n;
                exact_runs += need;
                if (n > kFastGiveUp) fast = false;
                if (count >= 32u) {
                    __syncwarp();
                    const uint2 e = ring[(head + (uint32_t)lane) & (kRing - 1u)];
                    __syncwarp();
                    head += 32u;
                    count -= 32u;
                    run_exact(e.x, e.y);
                }
            }
            // the rest of the tile on the exact path (after the warp gave the fast test up)
            for (; it < kPIPT; ++it) {
                if (pp < pend) {
                    if (pp >= nxt) {
                        while (pp >= s_off[jj + 1]) ++jj;
                        ci = s_id[jj];
                        ck = pp - s_off[jj];
                        nxt = s_off[jj + 1];
                    }
                    run_exact(ci, ck++);
                    ++pp;
                }
            }
            __syncwarp();
            if ((uint32_t)lane < count) {
                const uint2 q = ring[(head + (uint32_t)lane) & (kRing - 1u)];
                run_exact(q.x, q.y);
            }
        } else if (p < p1) {
            uint32_t pp = (uint32_t)p;
            // entry of particle pp in the window
            uint32_t a = 0, b = w;
            while (b - a > 1u) {
                uint32_t m = (a + b) >> 1;
                if (s_off[m] <= pp) a = m; else b = m;
            }
            uint32_t jj = a;
            uint32_t cur = 0xFFFFFFFFu;
            float4 R[kRecF4];
            const uint32_t pend = (uint32_t)(p + kPIPT < p1 ? p + kPIPT : p1);
            for (; pp < pend; ++pp) {
                while (pp >= s_off[jj + 1]) ++jj;
                const uint32_t i = s_id[jj];
                const uint32_t k = pp - s_off[jj];
                if (i != cur) {
                    cur = i;
                    const float4* Rg = rec + (size_t)i * kRecF4;
                    R[0] = __ldg(&Rg[0]);
                    R[1] = __ldg(&Rg[1]);
                    if (MC != 1) R[2] = __ldg(&Rg[2]);
                    if (MC == 1) {
                        R[2] = __ldg(&Rg[2]);
                        R[3] = __ldg(&Rg[3]);
                        R[4] = __ldg(&Rg[4]);
                        R[5] = __ldg(&Rg[5]);
                    }
                    if (MC == 2) R[3] = __ldg(&Rg[3]);
                }
                uint32_t rs = gx::particle_seed(i, k + 1u, seed);
                if (MC == 0) {
                    writes += emit_gps(f, T, s_lut, i, rs, R[0], R[1], R[2], S);
                } else if (MC == 1) {
                    uint32_t r;
                    if (FM == 0) {
                        r = emit_pbvr(f, T, i, rs, R, S);
                    } else {
                        const uint32_t q = pbvr_fast(f, rs, R);
                        if (FM == 2) {  // validation: always exact, count disagreements
                            r = emit_pbvr(f, T, i, rs, R, S);
                            mismatch += (q != 2u && q != r) ? 1u : 0u;
                        } else {
                            r = q == 2u ? emit_pbvr(f, T, i, rs, R, S) : q;
                        }
                        exact_runs += q == 2u ? 1u : 0u;
                    }
                    points += r & 1u;
                    writes += r >> 1;
                } else {
                    uint32_t r = emit_so(f, T, i, k, rs, R, S);
                    points += r;
                    writes += r;
                }
            }
        }
        // the first warp done with this tile finds the next one while the others still work
        uint32_t claim = 0u;
        if (lane == 0) claim = atomicExch(&s_claim, 1u);
        if (__shfl_sync(0xffffffffu, claim, 0) == 0u) find_unit();
        __syncthreads();
    }
    ull v = points, wv = writes, xv = exact_runs, mv = mismatch;
    for (int o = 16; o; o >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
        wv += __shfl_xor_sync(0xffffffffu, wv, o);
        xv += __shfl_xor_sync(0xffffffffu, xv, o);
        mv += __shfl_xor_sync(0xffffffffu, mv, o);
    }
    if (lane == 0 && v && MC != 0) atomicAdd(&stats[ST_POINTS], v);
    if (lane == 0 && wv) atomicAdd(&stats[ST_WRITES], wv);
    if (lane == 0 && xv) atomicAdd(&stats[ST_FAST_EXACT], xv);
    if (lane == 0 && mv) atomicAdd(&stats[ST_FAST_MISMATCH], mv);
}

template <int MC, int IPT, int FM>
static void launch_particles_t(const FrameConst& fc, const float4* rec, const float* lut, const uint2* clist,
                               const EnsTotal* etot, uint32_t first_seed, uint32_t E, unsigned long long* sub,
                               uint32_t* unit_counter, unsigned long long* stats, int grid, cudaStream_t st) {
    size_t smem = (kTabFloats + 2 * ((size_t)E + 1) + 2 * (kPT * IPT + 2)) * sizeof(uint32_t);
    if (MC == 0 && !fc.exact_radius) smem += kLutN * sizeof(float);
    if (MC == 1 && FM == 1) smem += (size_t)(kPT / 32) * kRing * sizeof(uint2);
    // the attribute belongs to each device's context: remember the size set per device ordinal
    static size_t attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    const bool known = dev >= 0 && dev < 64;
    if (smem > 48 * 1024 && (!known || smem > attr[dev])) {
        cudaFuncSetAttribute(k_particles<MC, IPT, FM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (known) attr[dev] = smem;
    }
    k_particles<MC, IPT, FM><<<grid, kPT, smem, st>>>(fc, rec, lut, clist, etot, first_seed, E, sub, unit_counter, stats);
}

template <int IPT>
static void launch_particles_m(const FrameConst& fc, const float4* rec, const float* lut, const uint2* clist,
                               const EnsTotal* etot, uint32_t first_seed, uint32_t E, unsigned long long* sub,
                               uint32_t* unit_counter, unsigned long long* stats, int grid, cudaStream_t st) {
    if (fc.method == 0u)
        launch_particles_t<0, IPT, 0>(fc, rec, lut, clist, etot, first_seed, E, sub, unit_counter, stats, grid, st);
    else if (fc.method == 4u)
        launch_particles_t<2, IPT, 0>(fc, rec, lut, clist, etot, first_seed, E, sub, unit_counter, stats, grid, st);
    else if (fc.fast_mode == 1u)
        launch_particles_t<1, IPT, 1>(fc, rec, lut, clist, etot, first_seed, E, sub, unit_counter, stats, grid, st);
    else if (fc.fast_mode == 2u)
        launch_particles_t<1, IPT, 2>(fc, rec, lut, clist, etot, first_seed, E, sub, unit_counter, stats, grid, st);
    else
        launch_particles_t<1, IPT, 0>(fc, rec, lut, clist, etot, first_seed, E, sub, unit_counter, stats, grid, st);
}

void launch_particles(const FrameConst& fc, const float4* rec, const float* lut, const uint2* clist,
                      const EnsTotal* etot, uint32_t first_seed, uint32_t E, unsigned long long* sub,
                      uint32_t* unit_counter, unsigned long long* stats, int grid, int items, cudaStream_t st) {
    cudaMemsetAsync(unit_counter, 0, sizeof(uint32_t), st);
    if (fc.N == 0 || E == 0) return;
    if (items >= 24)
        launch_particles_m<24>(fc, rec, lut, clist, etot, first_seed, E, sub, unit_counter, stats, grid, st);
    else if (items >= 16)
        launch_particles_m<16>(fc, rec, lut, clist, etot, first_seed, E, sub, unit_counter, stats, grid, st);
    else
        launch_particles_m<8>(fc, rec, lut, clist, etot, first_seed, E, sub, unit_counter, stats, grid, st);
}

// ============================================================================ primitive path
// splat_pass (gps_splat.wgsl:304-333): one thread per splat and ensemble generates all particles
// of the splat from one sequential stream. Validation path of GPS only (RenderPath::Primitive).
__global__ void __launch_bounds__(128) k_primitive(FrameConst f, const float4* __restrict__ rec,
                                                   const uint2* __restrict__ cdesc, const float* __restrict__ lut,
                                                   uint32_t first_seed, uint32_t E, ull* sub, ull* stats) {
    uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = gi % f.N, e = gi / f.N;
    if (e >= E) return;
    uint2 cd = __ldg(&cdesc[i]);
    if ((cd.y & 3u) != CD_POISSON_CAP) return;
    uint32_t rs = gx::particle_seed(i, 0u, first_seed + e);
    uint32_t n = poisson(__uint_as_float(cd.x), &rs);
    atomicAdd(&stats[ST_POINTS], (ull)n);
    atomicAdd(&stats[ST_VISIBLE], 1ull);
    if (n > f.cap) {
        atomicAdd(&stats[ST_TRUNCATED], 1ull);
        atomicAdd(&stats[ST_DROPPED], (ull)(n - f.cap));
        n = f.cap;
    }
    const float4* Rg = rec + (size_t)i * kRecF4;
    float4 r0 = Rg[0], r1 = Rg[1], r2 = Rg[2];
    ull* S = sub + (size_t)e * ((uint64_t)f.W * f.H * f.S);
    ull writes = 0;
    const FTabs T{gx::tab_log(), gx::tab_exp(), gx::tab_sc()};
    for (uint32_t q = 0; q < n; ++q) writes += emit_gps(f, T, lut, i, rs, r0, r1, r2, S);
    if (writes) atomicAdd(&stats[ST_WRITES], writes);
}

void launch_primitive(const FrameConst& fc, const float4* rec, const uint2* cdesc, const float* lut,
                      uint32_t first_seed, uint32_t E, unsigned long long* sub, EnsTotal* etot,
                      unsigned long long* stats, cudaStream_t st) {
    cudaMemsetAsync(etot, 0, (size_t)E * sizeof(EnsTotal), st);
    if (fc.N == 0 || E == 0) return;
    uint64_t n = (uint64_t)fc.N * E;
    k_primitive<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(fc, rec, cdesc, lut, first_seed, E, sub, stats);
}

// ============================================================================ resolve
// resolve (gps_splat.wgsl:362-386) for every ensemble of the batch, in ensemble order, so the
// f32 accumulation sequence equals the reference's one resolve per ensemble.
__global__ void __launch_bounds__(256) k_resolve(FrameConst f, const ull* __restrict__ sub,
                                                  const EnsTotal* __restrict__ etot, const float4* __restrict__ colour,
                                                  uint32_t E, float4* accum, ull* stats) {
    uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t P = f.W * f.H;
    if (pix >= P) return;
    const uint32_t S = f.S;
    const uint64_t PS = (uint64_t)P * S;
    float4 acc = accum[pix];
    const float inv_bg0 = f.bg[0], inv_bg1 = f.bg[1], inv_bg2 = f.bg[2];
    uint32_t orphans = 0;
    for (uint32_t e = 0; e < E; ++e) {
        if (__ldg(&etot[e].flags) != 0u) continue;
        const ull* s = sub + (size_t)e * PS + (size_t)pix * S;
        float sx = F_(0.0), sy = F_(0.0), sz = F_(0.0);
        for (uint32_t k = 0; k < S; ++k) {
            ull v = __ldcs(s + k);
            uint32_t key = (uint32_t)(v >> 32), id = (uint32_t)v;
            if (key == gxc::kEmpty) {
                sx = sx + inv_bg0; sy = sy + inv_bg1; sz = sz + inv_bg2;
            } else if (id == gxc::kEmpty) {
                ++orphans;
                sx = sx + inv_bg0; sy = sy + inv_bg1; sz = sz + inv_bg2;
            } else {
                float4 c = __ldg(&colour[id]);
                sx = sx + c.x; sy = sy + c.y; sz = sz + c.z;
            }
        }
        const float Sf = (float)S;
        acc.x = acc.x + div_(sx, Sf);
        acc.y = acc.y + div_(sy, Sf);
        acc.z = acc.z + div_(sz, Sf);
        acc.w = acc.w + F_(1.0);
    }
    accum[pix] = acc;
    if (orphans) atomicAdd(&stats[ST_ORPHAN], (ull)orphans);
}

void launch_resolve(const FrameConst& fc, const unsigned long long* sub, const EnsTotal* etot, const float4* colour,
                    uint32_t E, float4* accum, unsigned long long* stats, cudaStream_t st) {
    uint32_t P = fc.W * fc.H;
    if (P == 0 || E == 0) return;
    k_resolve<<<(P + 255) / 256, 256, 0, st>>>(fc, sub, etot, colour, E, accum, stats);
}

// Denoiser features of the batch's ensembles (no counterpart in the reference, which has no
// denoiser): per pixel and ensemble the resolved colour c (as k_resolve computes it), the covered
// fraction alpha of its subpixels and the covered subpixels' depth sum / S; adds (c.r^2, c.g^2,
// c.b^2, alpha, depth) to feat[pix * 8 + 0..4]. Skipped ensembles add nothing.
__global__ void __launch_bounds__(256) k_features(FrameConst f, const ull* __restrict__ sub,
                                                   const EnsTotal* __restrict__ etot, const float4* __restrict__ colour,
                                                   uint32_t E, float* feat) {
    uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t P = f.W * f.H;
    if (pix >= P) return;
    const uint32_t S = f.S;
    const uint64_t PS = (uint64_t)P * S;
    float q[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (uint32_t e = 0; e < E; ++e) {
        if (__ldg(&etot[e].flags) != 0u) continue;
        const ull* s = sub + (size_t)e * PS + (size_t)pix * S;
        float sx = F_(0.0), sy = F_(0.0), sz = F_(0.0), cov = 0.0f, dep = 0.0f;
        for (uint32_t k = 0; k < S; ++k) {
            ull v = __ldcs(s + k);
            uint32_t key = (uint32_t)(v >> 32), id = (uint32_t)v;
            if (key == gxc::kEmpty || id == gxc::kEmpty) {
                sx = sx + f.bg[0]; sy = sy + f.bg[1]; sz = sz + f.bg[2];
            } else {
                float4 c = __ldg(&colour[id]);
                sx = sx + c.x; sy = sy + c.y; sz = sz + c.z;
                cov += 1.0f;
                dep += __uint_as_float(key & 0x7FFFFFFFu);
            }
        }
        const float Sf = (float)S;
        const float cr = div_(sx, Sf), cg = div_(sy, Sf), cb = div_(sz, Sf);
        q[0] += cr * cr;
        q[1] += cg * cg;
        q[2] += cb * cb;
        q[3] += cov / Sf;
        q[4] += dep / Sf;
    }
    float* o = feat + (size_t)pix * 8;
#pragma unroll
    for (int j = 0; j < 5; ++j) o[j] += q[j];
}

void launch_features(const FrameConst& fc, const unsigned long long* sub, const EnsTotal* etot, const float4* colour,
                     uint32_t E, float* feat, cudaStream_t st) {
    const uint32_t P = fc.W * fc.H;
    if (P == 0 || E == 0) return;
    k_features<<<(P + 255) / 256, 256, 0, st>>>(fc, sub, etot, colour, E, feat);
}

__global__ void k_add_stat(ull* stats, int word, ull v) { stats[word] += v; }
void launch_add_stat(unsigned long long* stats, int word, unsigned long long v, cudaStream_t st) {
    k_add_stat<<<1, 1, 0, st>>>(stats, word, v);
}

// ----------------------------------------------------------------------------- debug probes
// The shared maths evaluated on the device, as the kernels evaluate it: which 0 exp, 1 log, 2 sin,
// 3 cos, 4 log for positive normal arguments, with the tables staged in shared memory (the
// particle kernel's form); which | 8: the same functions reading the global tables (the form of
// the other kernels).
__global__ void __launch_bounds__(256) k_debug_fmath(uint32_t which, const float* __restrict__ in,
                                                     float* __restrict__ out, uint64_t n) {
    __shared__ __align__(16) float s_tab[kTabFloats];
    const FTabs T = stage_tabs(s_tab);
    __syncthreads();
    const bool global = (which & 8u) != 0u;
    const uint32_t op = which & 7u;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float x = in[i];
        float y, sn, cs;
        if (op == 0u) {
            y = global ? gx::exp(x) : gx::exp_t(x, T.ex);
        } else if (op == 1u) {
            y = global ? gx::log(x) : gx::log_t(x, T.lg);
        } else if (op == 4u) {
            y = gx::log_t_pos(x, global ? gx::tab_log() : T.lg);
        } else {
            if (global) gx::sincos(x, &sn, &cs); else gx::sincos_t(x, T.sc, &sn, &cs);
            y = op == 2u ? sn : cs;
        }
        out[i] = y;
    }
}

void launch_debug_fmath(uint32_t which, const float* in, float* out, uint64_t n, cudaStream_t st) {
    if (n == 0) return;
    const uint64_t blocks = (n + 255) / 256;
    k_debug_fmath<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(which, in, out, n);
}

// For each particle p in [p0, p0 + n) of one ensemble's compact (splat id, offset) list: its splat
// i (the last entry with offset <= p, found with the particle kernel's 32-ary warp search), its
// index k within the splat and its stream seed particle_seed(i, k + 1, seed). out: 3 words per
// particle. One warp per 32 consecutive particles; the host checks p0 + n <= the list's total.
__global__ void __launch_bounds__(128) k_debug_seeds(const uint2* __restrict__ L, uint32_t nonzero, uint64_t p0,
                                                     uint32_t n, uint32_t seed, uint32_t* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u;
    if (base >= n) return;  // warp-uniform
    const uint32_t m = n - base < 32u ? n - base : 32u;
    for (uint32_t q = 0; q < m; ++q) {
        const uint64_t p = p0 + base + q;
        const uint32_t j = warp_last_le(L, 0u, nonzero, p, lane);
        if (lane == 0) {
            const uint2 e = L[j];
            const uint32_t k = (uint32_t)(p - e.y);
            out[3u * (base + q)] = e.x;
            out[3u * (base + q) + 1u] = k;
            out[3u * (base + q) + 2u] = gx::particle_seed(e.x, k + 1u, seed);
        }
    }
}

void launch_debug_seeds(const uint2* list, uint32_t nonzero, uint64_t p0, uint32_t n, uint32_t seed, uint32_t* out,
                        cudaStream_t st) {
    if (n == 0 || nonzero == 0) return;
    const uint32_t warps = (n + 31u) / 32u;
    k_debug_seeds<<<(warps + 3u) / 4u, 128, 0, st>>>(list, nonzero, p0, n, seed, out);
}

int device_sm_count(int device) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
    return n;
}

}  // namespace gpsb
