// O2: f32 mirror oracle of the reference GPU pipeline. TEST INFRASTRUCTURE ONLY.
//
// A sequential CPU restatement of shaders/gps_splat.wgsl (prepare / scan / finalize /
// particle passes / resolve / splat_pass / sp_project), shaders/gps_scan.wgsl,
// shaders/gps_sort.wgsl (stable order) and shaders/gps_composite.wgsl, evaluated exactly as
// the WGSL expressions read: every binary operator left to right with IEEE f32 rounding and no
// contraction (this file is compiled with -ffp-contract=off), WGSL abstract-float constants
// rounded once to f32, and exp/log/sin/cos taken from the shared deterministic fmath.h (WGSL
// leaves their precision implementation-defined). Integer RNG streams, seeds, counts and keys
// follow the shader bit for bit.
//
// The CUDA renderer is checked against this file for bit-exact counts, winners, statistics
// and accumulation. This file in turn is checked against O1 (the f64 gps-core restatement)
// with the reference's own statistical gates (crates/gps-render/src/verify.rs:120-123, 384-390).
//
// Deliberate, documented differences from the reference (shared with the CUDA renderer):
//   * the depth-sorted alpha path blends front to back in f32 with early termination at
//     transmittance < 1e-4 and evaluates the quad coordinates analytically per pixel centre
//     (the reference rasterises back-to-front quads into an rgba16f target,
//     gps_sorted_draw.wgsl:15-38, sorted.rs:125-138);
//   * the depth/colour two-pass atomicMin (gps_splat.wgsl:276-281) is evaluated here exactly as
//     two passes over the recorded particle writes; the CUDA side uses one 64-bit packed
//     atomicMin, which the parity tests show to be identical.
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <vector>
#include <algorithm>
#include <cmath>
#include <atomic>
#include <thread>

#include "../include/gpsb200.h"
#include "../gps-pbvr-web_b200/csrc/fmath.h"

using gx::fmax_;
using gx::fmin_;

namespace o2 {

struct V2 { float x, y; };
struct V3 { float x, y, z; };
struct V4 { float x, y, z, w; };

static inline float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 sub3(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 xyz(V4 a) { return {a.x, a.y, a.z}; }

// FrameUniform (crates/gps-render/src/gps.rs:61-76; shaders/gps_splat.wgsl:10-24)
struct Frame {
    V4 rot0, rot1, rot2, pos, intr;
    uint32_t dims[4], cfg[4], cfg2[4];
    V4 prm, bg;
    uint32_t pbvr[4];
    V4 pbp;
};

struct Scene {
    const gpsb_gaussian* g;
    uint32_t n;
    const float* sh;       // channel-major, sh_stride per channel
    uint32_t sh_stride;
    uint32_t sh_max_degree;
    const float* lut;      // 65 x 129
    double centroid[3];
};

static inline V4 gv(const gpsb_gaussian& g, int k) {
    const float* p = k == 0 ? g.pos_opacity : k == 1 ? g.log_scale : k == 2 ? g.rot_wxyz : g.color;
    return {p[0], p[1], p[2], p[3]};
}

// upload_frame (gps.rs:812-856)
static Frame make_frame(const Scene& s, const gpsb_camera& cam, const gpsb_params& p, uint32_t W,
                        uint32_t H, uint32_t side, uint32_t seed) {
    Frame f;
    memset(&f, 0, sizeof f);
    const double* R = cam.view_rot;
    f.rot0 = {(float)R[0], (float)R[1], (float)R[2], (float)0.0};
    f.rot1 = {(float)R[3], (float)R[4], (float)R[5], (float)0.0};
    f.rot2 = {(float)R[6], (float)R[7], (float)R[8], (float)0.0};
    f.pos = {(float)cam.view_pos[0], (float)cam.view_pos[1], (float)cam.view_pos[2], (float)cam.low_pass};
    double cx = cam.cx, cy = cam.cy;
    if (cam.cx == 0.0 && cam.cy == 0.0) { cx = 0.5 * W; cy = 0.5 * H; }
    f.intr = {(float)cam.focal_x, (float)cam.focal_y, (float)cx, (float)cy};
    f.dims[0] = W; f.dims[1] = H; f.dims[2] = side; f.dims[3] = s.n;
    f.cfg[0] = seed;
    f.cfg[1] = p.max_points_per_splat > 1 ? p.max_points_per_splat : 1;
    f.cfg2[1] = s.sh_stride;
    f.cfg2[2] = p.exact_radius ? 1u : 0u;
    f.prm = {p.density_scale, p.near_z, (float)0.0, (float)0.0};
    f.bg = {p.background[0], p.background[1], p.background[2], (float)0.0};
    uint32_t flags = (p.pbvr.radial_correction ? 1u : 0u) | (p.pbvr.centre_depth ? 2u : 0u) |
                     (p.pbvr.low_pass_jitter ? 4u : 0u);
    f.pbvr[0] = p.method;
    f.pbvr[1] = p.pbvr.calibration;
    f.pbvr[2] = flags;
    f.pbvr[3] = std::min(p.sh_degree, s.sh_max_degree);
    double d[3] = {s.centroid[0] - cam.view_pos[0], s.centroid[1] - cam.view_pos[1], s.centroid[2] - cam.view_pos[2]};
    double od = R[6] * d[0] + R[7] * d[1] + R[8] * d[2];
    f.pbp = {p.pbvr.base_k, p.pbvr.reference_pixel_length, (float)od, (float)0.0};
    return f;
}

struct Stats {  // 64-bit counters, reference word order (gps_splat.wgsl:38-44)
    uint64_t c[16];
};

// ----------------------------------------------------------------------- Li2 (gps_splat.wgsl:79-140)
static float dilog_series(float x) {
    float term = x, sum = x;
    for (uint32_t k = 2; k < 32; ++k) {
        term = term * x;
        sum = sum + gx::div_(term, (float)(k * k));
    }
    return sum;
}
static float dilog(float x) {
    if (x >= (float)1.0) return gxc::kDilogOne;
    if (x <= (float)0.0) return (float)0.0;
    if (x <= (float)0.5) return dilog_series(x);
    return gxc::kDilogOne - gx::log(x) * gx::log((float)1.0 - x) - dilog_series((float)1.0 - x);
}
static float inv_dilog(float tgt, float hi_in) {
    if (tgt <= (float)0.0) return (float)0.0;
    float lo = (float)0.0, hi = hi_in, y = hi * (float)0.5;
    for (uint32_t i = 0; i < 24; ++i) {
        float f = dilog(y) - tgt;
        if (f > (float)0.0) hi = y; else lo = y;
        float dfdy = (float)1.0;
        if (y > (float)1e-6 && y < (float)0.9999999) dfdy = gx::div_(-gx::log((float)1.0 - y), y);
        float ny = y - gx::div_(f, dfdy);
        if (!(ny > lo && ny < hi)) ny = (float)0.5 * (lo + hi);
        if (fabsf(ny - y) <= (float)1e-6 * ((float)1.0 + y)) return ny;
        y = ny;
    }
    return y;
}
static inline float mix(float a, float b, float t) { return a * ((float)1.0 - t) + b * t; }
static float corrected_radius_lut(const float* lut, float o, float u) {
    if (o <= (float)0.0) return (float)0.0;
    float v = -gx::log(fmax_((float)1.0 - u, gxc::kUMin));
    float fo = ((float)1.0 - gx::sqrt_(fmax_((float)1.0 - fmin_(o, (float)1.0), (float)0.0))) * (float)64.0;
    float fv = fmin_(gx::sqrt_(v) * gxc::kLutFv, (float)128.0);
    uint32_t i0 = std::min(gx::f2u(fo), 63u), j0 = std::min(gx::f2u(fv), 127u);
    float a = fo - (float)i0, b = fv - (float)j0;
    uint32_t k = i0 * 129u + j0;
    float r0 = mix(lut[k], lut[k + 1], b);
    float r1 = mix(lut[k + 129], lut[k + 130], b);
    return mix(r0, r1, a);
}
static float corrected_radius(float o, float u) {
    if (o <= (float)0.0) return (float)0.0;
    float d = dilog(o);
    float tgt = ((float)1.0 - u) * d;
    float y = fmin_(inv_dilog(tgt, o), o);
    if (y <= (float)0.0) return (float)40.0;
    return gx::sqrt_(fmax_(-(float)2.0 * gx::log(gx::div_(y, o)), (float)0.0));
}

// ----------------------------------------------------------------------- RNG helpers
struct Rng {
    uint32_t st;
    bool has_spare;
    float spare;
    float next() { return gx::next_u(&st); }
    // normal() (gps_splat.wgsl:402-414)
    float normal() {
        if (has_spare) { has_spare = false; return spare; }
        float u1 = fmax_(next(), gxc::kUMin);
        float u2 = next();
        float r = gx::sqrt_(-(float)2.0 * gx::log(u1));
        float th = gxc::kTwoPi * u2;
        float sn, cs;
        gx::sincos(th, &sn, &cs);
        spare = r * sn;
        has_spare = true;
        return r * cs;
    }
};

// poisson (gps_splat.wgsl:142-160)
static uint32_t poisson(float lambda, Rng& rng) {
    if (lambda <= (float)0.0) return 0u;
    if (lambda < (float)30.0) {
        float l = gx::exp(-lambda);
        uint32_t k = 0;
        float p = (float)1.0;
        for (;;) {
            k = k + 1u;
            p = p * rng.next();
            if (p <= l) break;
        }
        return k - 1u;
    }
    float u1 = fmax_(rng.next(), gxc::kUMin);
    float u2 = rng.next();
    float z = gx::sqrt_(-(float)2.0 * gx::log(u1)) * gx::cos(gxc::kTwoPi * u2);
    return gx::f2u(fmax_(gx::rint_(lambda + gx::sqrt_(lambda) * z), (float)0.0));
}

// ----------------------------------------------------------------------- projection (gps_splat.wgsl:165-206)
struct Proj { bool ok; float mx, my, a, b, c, depth; };

static void rot_cols(V4 q0, V3& c0, V3& c1, V3& c2) {
    float len = gx::sqrt_(q0.x * q0.x + q0.y * q0.y + q0.z * q0.z + q0.w * q0.w);
    float w = gx::div_(q0.x, len), x = gx::div_(q0.y, len), y = gx::div_(q0.z, len), z = gx::div_(q0.w, len);
    c0 = {(float)1.0 - (float)2.0 * (y * y + z * z), (float)2.0 * (x * y + w * z), (float)2.0 * (x * z - w * y)};
    c1 = {(float)2.0 * (x * y - w * z), (float)1.0 - (float)2.0 * (x * x + z * z), (float)2.0 * (y * z + w * x)};
    c2 = {(float)2.0 * (x * z + w * y), (float)2.0 * (y * z - w * x), (float)1.0 - (float)2.0 * (x * x + y * y)};
}

static Proj project(const Frame& f, const gpsb_gaussian& g) {
    Proj pr;
    pr.ok = false;
    V4 g0 = gv(g, 0), g1 = gv(g, 1), g2 = gv(g, 2);
    V3 p = sub3(xyz(g0), xyz(f.pos));
    V3 cam = {dot3(xyz(f.rot0), p), dot3(xyz(f.rot1), p), dot3(xyz(f.rot2), p)};
    if (cam.z <= fmax_(f.prm.y, (float)1e-4)) return pr;
    float lim = gxc::kFrustumLim;
    float tx = gx::clamp_(gx::div_(cam.x, cam.z), -lim, lim) * cam.z;
    float ty = gx::clamp_(gx::div_(cam.y, cam.z), -lim, lim) * cam.z;
    float fx = f.intr.x, fy = f.intr.y;
    float iz = gx::div_((float)1.0, cam.z);
    float s0 = fx * iz, s1 = -fx * tx * iz * iz;
    float s2 = fy * iz, s3 = -fy * ty * iz * iz;
    V3 m0 = {f.rot0.x * s0 + f.rot2.x * s1, f.rot0.y * s0 + f.rot2.y * s1, f.rot0.z * s0 + f.rot2.z * s1};
    V3 m1 = {f.rot1.x * s2 + f.rot2.x * s3, f.rot1.y * s2 + f.rot2.y * s3, f.rot1.z * s2 + f.rot2.z * s3};
    V3 c0, c1, c2;
    rot_cols(g2, c0, c1, c2);
    V3 sc = {gx::exp((float)2.0 * g1.x), gx::exp((float)2.0 * g1.y), gx::exp((float)2.0 * g1.z)};
    V3 u = {dot3(m0, c0), dot3(m0, c1), dot3(m0, c2)};
    V3 v = {dot3(m1, c0), dot3(m1, c1), dot3(m1, c2)};
    float a = dot3(sc, {u.x * u.x, u.y * u.y, u.z * u.z}) + f.pos.w;
    float b = dot3(sc, {u.x * v.x, u.y * v.y, u.z * v.z});
    float c = dot3(sc, {v.x * v.x, v.y * v.y, v.z * v.z}) + f.pos.w;
    float det = a * c - b * b;
    if (!(det > (float)0.0)) return pr;
    pr.ok = true;
    pr.mx = gx::div_(fx * cam.x, cam.z) + f.intr.z;
    pr.my = gx::div_(fy * cam.y, cam.z) + f.intr.w;
    pr.a = a; pr.b = b; pr.c = c;
    pr.depth = cam.z;
    return pr;
}

// splat_colour (gps_splat.wgsl:210-251)
static V3 splat_colour(const Frame& f, const Scene& s, uint32_t id) {
    V4 base4 = gv(s.g[id], 3);
    V3 res = {base4.x, base4.y, base4.z};
    uint32_t deg = f.pbvr[3];
    if (deg == 0u) return {fmax_(res.x, (float)0.0), fmax_(res.y, (float)0.0), fmax_(res.z, (float)0.0)};
    V4 p4 = gv(s.g[id], 0);
    V3 dv = sub3(xyz(p4), xyz(f.pos));
    float len = gx::sqrt_(dot3(dv, dv));
    float x = gx::div_(dv.x, len), y = gx::div_(dv.y, len), z = gx::div_(dv.z, len);
    uint32_t r = s.sh_stride;
    const float* sh = s.sh + (size_t)id * 3u * r;
    auto S = [&](uint32_t k, int ch) { return sh[ch * r + k]; };
    float out[3];
    for (int ch = 0; ch < 3; ++ch) {
        float acc = ch == 0 ? res.x : ch == 1 ? res.y : res.z;
        acc = acc - (float)0.488602519 * y * S(0, ch) + (float)0.488602519 * z * S(1, ch) - (float)0.488602519 * x * S(2, ch);
        if (deg >= 2u) {
            float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            acc = acc + (float)1.09254849 * xy * S(3, ch) - (float)1.09254849 * yz * S(4, ch) +
                  (float)0.31539157 * ((float)2.0 * zz - xx - yy) * S(5, ch) - (float)1.09254849 * xz * S(6, ch) +
                  (float)0.546274215 * (xx - yy) * S(7, ch);
            if (deg >= 3u) {
                acc = acc - (float)0.590043604 * y * ((float)3.0 * xx - yy) * S(8, ch) + (float)2.89061141 * xy * z * S(9, ch) -
                      (float)0.457045794 * y * ((float)4.0 * zz - xx - yy) * S(10, ch) +
                      (float)0.373176336 * z * ((float)2.0 * zz - (float)3.0 * xx - (float)3.0 * yy) * S(11, ch) -
                      (float)0.457045794 * x * ((float)4.0 * zz - xx - yy) * S(12, ch) +
                      (float)1.44530571 * z * (xx - yy) * S(13, ch) - (float)0.590043604 * x * (xx - (float)3.0 * yy) * S(14, ch);
            }
        }
        out[ch] = fmax_(acc, (float)0.0);
    }
    return {out[0], out[1], out[2]};
}

// ----------------------------------------------------------------------- renderer state
struct Write { uint32_t idx, key, id; };

// (key << 32) | id of a subpixel written by one of several threads: the minimum packed word is the
// minimum depth key and, among equal keys, the minimum splat id, the same winner as the two passes
// over the recorded writes (the single-threaded form below).
static inline void packed_min(std::atomic<uint64_t>& w, uint64_t v) {
    uint64_t cur = w.load(std::memory_order_relaxed);
    while (v < cur && !w.compare_exchange_weak(cur, v, std::memory_order_relaxed)) {
    }
}

struct Pipeline {
    const Scene& s;
    Frame f;
    uint32_t W, H, side, S;
    V4* proj = nullptr;              // 6 x vec4 per splat (storage owned by the caller)
    std::vector<Write> writes;       // particle writes of the depth pass, replayed by the colour pass
    std::atomic<uint64_t>* packed = nullptr;  // threaded form: writes go straight to the packed words
    uint64_t nwrites = 0;            // writes of the threaded form
    Stats& st;
    uint64_t running;                // stats[8] as an exact 64-bit running total
    bool overflow;                   // stats[9]

    Pipeline(const Scene& sc, Stats& stt) : s(sc), st(stt) {}

    bool offscreen(const Proj& pr) const {
        float ex = gxc::kOffscreenSigma * gx::sqrt_(pr.a);
        float ey = gxc::kOffscreenSigma * gx::sqrt_(pr.c);
        return pr.mx + ex < (float)0.0 || pr.mx - ex >= (float)W || pr.my + ey < (float)0.0 || pr.my - ey >= (float)H;
    }
    float expected_count(const Proj& pr, float o) const {
        float det = pr.a * pr.c - pr.b * pr.b;
        return f.prm.x * (float)S * (float)2.0 * gxc::kPi * gx::sqrt_(det) * dilog(o);
    }
    void write_key(uint32_t idx, uint32_t key, uint32_t id) {
        if (packed) {
            packed_min(packed[idx], ((uint64_t)key << 32) | id);
            ++nwrites;
        } else {
            writes.push_back({idx, key, id});
        }
    }
    void write(uint32_t idx, float depth_z, uint32_t id) { write_key(idx, gx::f2b(depth_z) | 0x80000000u, id); }

    // emit_particle (gps_splat.wgsl:259-282)
    void emit_gps(uint32_t gid, Rng& rng, float mx, float my, float depth_z, float o, float l00, float l10, float l11) {
        float r = f.cfg2[2] == 0u ? corrected_radius_lut(s.lut, o, rng.next()) : corrected_radius(o, rng.next());
        float th = gxc::kTwoPi * rng.next();
        float sn, cs;
        gx::sincos(th, &sn, &cs);
        float wx = r * cs, wy = r * sn;
        float px_ = mx + l00 * wx;
        float py_ = my + (l10 * wx + l11 * wy);
        if (px_ < (float)0.0 || px_ >= (float)W || py_ < (float)0.0 || py_ >= (float)H) return;
        uint32_t px = gx::f2u(px_), py = gx::f2u(py_);
        uint32_t sx = std::min(side - 1u, gx::f2u((px_ - (float)px) * (float)side));
        uint32_t sy = std::min(side - 1u, gx::f2u((py_ - (float)py) * (float)side));
        write((py * W + px) * S + sy * side + sx, depth_z, gid);
    }

    // pixel_density_scale / extinction_term / radial_keep / pbvr_lambda (gps_splat.wgsl:417-460)
    float pds(float depth) const {
        if (!(depth > fmax_(f.prm.y, (float)0.0))) return (float)0.0;
        float ratio = gx::div_(f.pbp.y, depth);
        return fmin_(ratio * ratio * f.intr.x * f.intr.y, (float)1.0e12);
    }
    static float extinction_term(float o) {
        float c = fmin_(o, gxc::kOneMinus1e6);
        if (c < (float)1e-3) return c * ((float)1.0 + c * ((float)0.5 + c * (float)0.33333334));
        return -gx::log((float)1.0 - c);
    }
    static float eol(float x) {
        if (x < (float)1e-4) return (float)1.0 + (float)0.5 * x;
        return gx::div_(-gx::log((float)1.0 - fmin_(x, gxc::kOneMinus1e6)), x);
    }
    static float radial_keep(float o, float r2) {
        float oo = fmin_(o, gxc::kOneMinus1e6);
        float y = oo * gx::exp(-(float)0.5 * fmax_(r2, (float)0.0));
        return gx::clamp_(gx::div_(eol(y), eol(oo)), (float)0.0, (float)1.0);
    }
    float pbvr_lambda(const Proj& pr, float o) const {
        uint32_t method = f.pbvr[0];
        float g = extinction_term(o);
        if (method == 1u) g = fmin_(o, gxc::kOneMinus1e6);
        float scale = f.pbp.x;
        if (method != 3u) {
            uint32_t level = f.pbvr[1];
            if (level == 1u) scale = scale * pds(f.pbp.z);
            else if (level == 2u) scale = scale * pds(pr.depth);
            else if (level == 3u) scale = (float)S * (float)2.0 * gxc::kPi * gx::sqrt_(pr.a * pr.c - pr.b * pr.b);
        }
        float n = f.prm.x * g * scale;
        if (!(n > (float)0.0) || n > (float)3.0e38) return (float)0.0;
        return n;
    }

    // chol_of (gps_splat.wgsl:464-485)
    void chol_of(uint32_t gid, V3& ca, V3& cb) const {
        V4 g1 = gv(s.g[gid], 1);
        V3 c0, c1, c2;
        rot_cols(gv(s.g[gid], 2), c0, c1, c2);
        V3 s2 = {gx::exp((float)2.0 * g1.x), gx::exp((float)2.0 * g1.y), gx::exp((float)2.0 * g1.z)};
        float a00 = s2.x * c0.x * c0.x + s2.y * c1.x * c1.x + s2.z * c2.x * c2.x;
        float a10 = s2.x * c0.y * c0.x + s2.y * c1.y * c1.x + s2.z * c2.y * c2.x;
        float a20 = s2.x * c0.z * c0.x + s2.y * c1.z * c1.x + s2.z * c2.z * c2.x;
        float a11 = s2.x * c0.y * c0.y + s2.y * c1.y * c1.y + s2.z * c2.y * c2.y;
        float a21 = s2.x * c0.z * c0.y + s2.y * c1.z * c1.y + s2.z * c2.z * c2.y;
        float a22 = s2.x * c0.z * c0.z + s2.y * c1.z * c1.z + s2.z * c2.z * c2.z;
        float l00 = gx::sqrt_(fmax_(a00, (float)1e-30));
        float l10 = gx::div_(a10, l00);
        float l20 = gx::div_(a20, l00);
        float l11 = gx::sqrt_(fmax_(a11 - l10 * l10, (float)1e-30));
        float l21 = gx::div_(a21 - l20 * l10, l11);
        float l22 = gx::sqrt_(fmax_(a22 - l20 * l20 - l21 * l21, (float)1e-30));
        ca = {l00, l10, l11};
        cb = {l20, l21, l22};
    }

    // emit_particle_pbvr (gps_splat.wgsl:490-532): the answer of particle `rng`, 0 = not a point,
    // 1 = a point off screen, 3 = a point written to subpixel idx at depth_z
    uint32_t pbvr_eval(Rng& rng, V4 a, V4 b, V4 c, V4 d, V3 ca, V3 cb, uint32_t& idx, float& depth_z) {
        rng.has_spare = false;
        float uz = rng.normal();
        float uy = rng.normal();
        float ux = rng.normal();
        if (f.pbvr[0] == 3u) {
            if (rng.next() >= b.w) return 0u;
        }
        V3 world = {c.x + ca.x * ux, c.y + (ca.y * ux + ca.z * uy), c.z + (cb.x * ux + cb.y * uy + cb.z * uz)};
        V3 p = sub3(world, xyz(f.pos));
        V3 cam = {dot3(xyz(f.rot0), p), dot3(xyz(f.rot1), p), dot3(xyz(f.rot2), p)};
        if (cam.z <= f.prm.y) return 0u;
        float pix_x = gx::div_(f.intr.x * cam.x, cam.z) + f.intr.z;
        float pix_y = gx::div_(f.intr.y * cam.y, cam.z) + f.intr.w;
        uint32_t flags = f.pbvr[2];
        if (flags & 4u) {
            float jy = rng.normal();
            float jx = rng.normal();
            float sj = gx::sqrt_(fmax_(f.pos.w, (float)0.0));
            pix_x = pix_x + sj * jx;
            pix_y = pix_y + sj * jy;
        }
        if (flags & 1u) {
            float dvx = pix_x - a.x, dvy = pix_y - a.y;
            float r2 = c.w * dvx * dvx + (float)2.0 * d.x * dvx * dvy + d.y * dvy * dvy;
            if (rng.next() >= radial_keep(a.w, r2)) return 0u;
        }
        depth_z = cam.z;
        if (flags & 2u) depth_z = a.z;
        if (pix_x < (float)0.0 || pix_x >= (float)W || pix_y < (float)0.0 || pix_y >= (float)H) return 1u;
        uint32_t px = gx::f2u(pix_x), py = gx::f2u(pix_y);
        uint32_t sx = std::min(side - 1u, gx::f2u((pix_x - (float)px) * (float)side));
        uint32_t sy = std::min(side - 1u, gx::f2u((pix_y - (float)py) * (float)side));
        idx = (py * W + px) * S + sy * side + sx;
        return 3u;
    }
    void emit_pbvr(uint32_t gid, Rng& rng, V4 a, V4 b, V4 c, V4 d, V3 ca, V3 cb) {
        uint32_t idx = 0;
        float depth_z = (float)0.0;
        const uint32_t r = pbvr_eval(rng, a, b, c, d, ca, cb, idx, depth_z);
        if (r & 1u) st.c[0] += 1;  // points (depth pass only)
        if (r == 3u) write(idx, depth_z, gid);
    }

    uint32_t prepare_gps(uint32_t i, const Proj& pr, float o) {
        if (offscreen(pr)) return 0u;
        float en = expected_count(pr, o);
        if (!(en > (float)0.0)) return 0u;
        Rng rng{gx::particle_seed(i, 0u, f.cfg[0]), false, (float)0.0};
        uint32_t n = poisson(en, rng);
        st.c[0] += n;
        st.c[3] += 1;
        uint32_t cap = f.cfg[1];
        if (n > cap) { st.c[1] += 1; st.c[2] += n - cap; n = cap; }
        return n;
    }

    uint32_t prepare_pbvr(uint32_t i, const Proj& pr, float o) {
        V4* P = &proj[(size_t)i * 6u];
        if (f.pbvr[0] == 4u) {
            float density = fmax_(f.prm.x, (float)1e-8);
            float amin = fmax_((float)1.0 - gx::exp(gx::div_(gxc::kLn254over255, density)), (float)1e-8);
            if (o <= amin) return 0u;
            float radius = gx::sqrt_((float)2.0 * gx::log(gx::div_(o, amin)));
            float ext_x = radius * gx::sqrt_(pr.a), ext_y = radius * gx::sqrt_(pr.c);
            float lo_x = gx::clamp_(floorf(pr.mx - ext_x), (float)0.0, (float)W);
            float lo_y = gx::clamp_(floorf(pr.my - ext_y), (float)0.0, (float)H);
            float hi_x = gx::clamp_(ceilf(pr.mx + ext_x), (float)0.0, (float)W);
            float hi_y = gx::clamp_(ceilf(pr.my + ext_y), (float)0.0, (float)H);
            float sz_x = fmax_(hi_x - lo_x, (float)0.0), sz_y = fmax_(hi_y - lo_y, (float)0.0);
            uint32_t count = gx::f2u(sz_x) * gx::f2u(sz_y) * side * side;
            if (count == 0u) return 0u;
            float invdet = gx::div_((float)1.0, fmax_(pr.a * pr.c - pr.b * pr.b, (float)1e-30));
            P[1] = {lo_x, lo_y, sz_x, sz_y};
            float peak_tau = -gx::log((float)1.0 - fmin_(o, gxc::kOneMinus1e6));
            bool sparse = density * peak_tau < (float)1.0;
            uint32_t trials = count;
            if (sparse) {
                Rng rng{gx::particle_seed(i, 0u, f.cfg[0]), false, (float)0.0};
                trials = poisson((float)count * density * peak_tau, rng);
            }
            P[2] = {pr.c * invdet, -pr.b * invdet, pr.a * invdet, peak_tau};
            P[3].w = sparse ? (float)1.0 : (float)0.0;
            st.c[5] += trials;
            st.c[3] += 1;
            return trials;
        }
        float lambda = pbvr_lambda(pr, o);
        if (!(lambda > (float)0.0)) return 0u;
        float det = pr.a * pr.c - pr.b * pr.b;
        float keep = (float)1.0;
        if (f.pbvr[0] == 3u) {
            float target = f.prm.x * (float)S * (float)2.0 * gxc::kPi * gx::sqrt_(det) * dilog(o);
            if (lambda > (float)0.5) keep = gx::clamp_(gx::div_(target, lambda), (float)0.0, (float)1.0); else keep = (float)0.0;
            if (target > lambda) st.c[6] += 1;
        }
        Rng rng{gx::particle_seed(i, 0u, f.cfg[0]), false, (float)0.0};
        uint32_t n = poisson(lambda, rng);
        st.c[5] += n;
        st.c[3] += 1;
        uint32_t cap = f.cfg[1];
        if (n > cap) { st.c[1] += 1; st.c[2] += n - cap; n = cap; }
        float idet = gx::div_((float)1.0, fmax_(det, (float)1e-30));
        V4 g0 = gv(s.g[i], 0);
        P[1].w = keep;
        P[2] = {g0.x, g0.y, g0.z, pr.c * idet};
        P[3] = {-pr.b * idet, pr.a * idet, (float)0.0, (float)0.0};
        V3 ca, cb;
        chol_of(i, ca, cb);
        P[4] = {ca.x, ca.y, ca.z, (float)0.0};
        P[5] = {cb.x, cb.y, cb.z, (float)0.0};
        return n;
    }

    // prepare (gps_splat.wgsl:617-642)
    uint32_t prepare(uint32_t i) {
        uint32_t cnt = 0;
        Proj pr = project(f, s.g[i]);
        float o = gx::clamp_(s.g[i].pos_opacity[3], (float)0.0, (float)1.0);
        if (pr.ok && o > (float)0.0) {
            float l00 = gx::sqrt_(fmax_(pr.a, (float)1e-30));
            float l10 = gx::div_(pr.b, l00);
            float l11 = gx::sqrt_(fmax_(pr.c - l10 * l10, (float)1e-30));
            proj[(size_t)i * 6u] = {pr.mx, pr.my, pr.depth, o};
            proj[(size_t)i * 6u + 1u] = {l00, l10, l11, (float)1.0};
            cnt = f.pbvr[0] == 0u ? prepare_gps(i, pr, o) : prepare_pbvr(i, pr, o);
        }
        if (cnt > 0u) {
            // exact u32 overflow detection of the scan total (gps_splat.wgsl:635-639)
            if (running + cnt > 0xFFFFFFFFull) overflow = true;
            running += cnt;
        }
        return cnt;
    }

    // particle_pass (gps_splat.wgsl:677-714) for particle (i, k)
    void particle(uint32_t i, uint32_t k) {
        V4 a = proj[(size_t)i * 6u], b = proj[(size_t)i * 6u + 1u];
        Rng rng{gx::particle_seed(i, k + 1u, f.cfg[0]), false, (float)0.0};
        if (f.pbvr[0] == 4u) {
            uint32_t samples = side * side;
            bool sparse = proj[(size_t)i * 6u + 3u].w > (float)0.0;
            uint32_t cell = k;
            uint32_t bz = gx::f2u(b.z), bw = gx::f2u(b.w);
            if (sparse) cell = std::min(gx::f2u(rng.next() * b.z * b.w * (float)samples), bz * bw * samples - 1u);
            uint32_t pixel = cell / samples, sub = cell % samples;
            uint32_t xx = gx::f2u(b.x) + pixel % bz, yy = gx::f2u(b.y) + pixel / bz;
            float n1 = rng.next();
            float n2 = rng.next();
            float uvx = gx::div_((float)(sub % side) + n1, (float)side);
            float uvy = gx::div_((float)(sub / side) + n2, (float)side);
            float dx = (float)xx + uvx - a.x, dy = (float)yy + uvy - a.y;
            V4 inv = proj[(size_t)i * 6u + 2u];
            float r2 = fmax_(inv.x * dx * dx + (float)2.0 * inv.y * dx * dy + inv.z * dy * dy, (float)0.0);
            float alpha = fmin_(a.w * gx::exp(-(float)0.5 * r2), gxc::kOneMinus1e6);
            float coverage = (float)1.0 - gx::exp(f.prm.x * gx::log((float)1.0 - alpha));
            if (sparse) coverage = gx::div_(-gx::log((float)1.0 - alpha), inv.w);
            if (rng.next() >= coverage) return;
            uint32_t idx = (yy * W + xx) * samples + sub;
            st.c[0] += 1;
            write_key(idx, gx::f2b(a.z) | 0x80000000u, i);
        } else if (f.pbvr[0] == 0u) {
            emit_gps(i, rng, a.x, a.y, a.z, a.w, b.x, b.y, b.z);
        } else {
            V4 c = proj[(size_t)i * 6u + 2u], d = proj[(size_t)i * 6u + 3u];
            V4 e4 = proj[(size_t)i * 6u + 4u], f4 = proj[(size_t)i * 6u + 5u];
            emit_pbvr(i, rng, a, b, c, d, {e4.x, e4.y, e4.z}, {f4.x, f4.y, f4.z});
        }
    }

    // splat_pass (gps_splat.wgsl:304-333), primitive path, GPS only
    void splat_pass(uint32_t gid) {
        Proj pr = project(f, s.g[gid]);
        if (!pr.ok) return;
        float o = gx::clamp_(s.g[gid].pos_opacity[3], (float)0.0, (float)1.0);
        if (o <= (float)0.0) return;
        if (offscreen(pr)) return;
        float en = expected_count(pr, o);
        if (!(en > (float)0.0)) return;
        Rng rng{gx::particle_seed(gid, 0u, f.cfg[0]), false, (float)0.0};
        uint32_t n = poisson(en, rng);
        st.c[0] += n;
        st.c[3] += 1;
        uint32_t cap = f.cfg[1];
        if (n > cap) { st.c[1] += 1; st.c[2] += n - cap; n = cap; }
        float l00 = gx::sqrt_(fmax_(pr.a, (float)1e-30));
        float l10 = gx::div_(pr.b, l00);
        float l11 = gx::sqrt_(fmax_(pr.c - l10 * l10, (float)1e-30));
        for (uint32_t i = 0; i < n; ++i) emit_gps(gid, rng, pr.mx, pr.my, pr.depth, o, l00, l10, l11);
    }
};


// ----------------------------------------------------------------------- fast-decision check
// A restatement of the renderer's PBVR fast decisions (pbvr_fast, fast_pair and fast_bounds_of in
// gps-pbvr-web_b200/csrc/kernels.cu, line for line) in which every hardware approximation is
// replaced by the exact value pushed to the edge of the error bound the decisions assume:
// log by +-(kLogAbs + kLogRel |log|), the Box-Muller radius by +-kErMax, sin and cos by
// +-kSinCos, exp by a relative +-(kExpA + kExpB |a|), reciprocals by +-2^-23 relative (signs
// random per operand, or all + / all -). Whenever the restated fast path answers "not a point"
// or "a point off screen", the exact path (pbvr_eval) must agree: this checks the error
// propagation of the decisions on the CPU, independently of the device's approximations (whose
// constants the renderer checks exhaustively on the GPU).
namespace fastcheck {
constexpr float kU = 6.0e-8f, kSafe = 1.01f;
constexpr float kLogAbs = 3.5e-7f, kLogRel = 3.5e-7f, kSinCos = 1e-6f, kXMin = 1e-3f, kErMax = 2.5e-6f;
constexpr float kRMax = 5.77f;
constexpr float kEN = kErMax * (1.0f + 2.0f * kSinCos) + kRMax * (kSinCos + 2.01f * kU) + 1e-7f;
constexpr float kExpA = 6e-7f, kExpB = 1.5e-7f, kExpTiny = 1.5e-38f;
constexpr float kEdge = 0.999f;  // how far to the edge of each bound the perturbations go

struct Perturb {
    uint32_t st;
    int mode;  // 0 random signs, 1 all +, 2 all -
    float sgn() {
        if (mode == 1) return 1.0f;
        if (mode == 2) return -1.0f;
        st = gx::pcg(st);
        return (st >> 16) & 1u ? 1.0f : -1.0f;
    }
    float log_(float v) {
        const float e = gx::log(v);
        return e + sgn() * (kLogAbs + kLogRel * fabsf(e)) * kEdge;
    }
    float exp_(float a) {
        const double e = (double)gx::exp(a);
        return (float)(e * (1.0 + sgn() * (kExpA + kExpB * fabs((double)a)) * kEdge));
    }
    float rcp_(float x) { return (float)((1.0 / (double)x) * (1.0 + sgn() * 1.19e-7 * kEdge)); }
};

struct Bounds { float fx_ecx, fy_ecy, ecz, kq, gx_, gy_; };

// fast_bounds_of
static Bounds bounds_of(const Frame& f, V3 g0, V3 ca, V3 cb, float a, float b, float c) {
    const float sx = fabsf(ca.x), sy = fabsf(ca.y) + fabsf(ca.z), sz = fabsf(cb.x) + fabsf(cb.y) + fabsf(cb.z);
    const float gm = kRMax + kEN;
    const float Mx = fabsf(g0.x) + fabsf(f.pos.x) + sx * gm, My = fabsf(g0.y) + fabsf(f.pos.y) + sy * gm,
                Mz = fabsf(g0.z) + fabsf(f.pos.z) + sz * gm;
    const float ex = sx * kEN + 6.0f * kU * Mx, ey = sy * kEN + 10.0f * kU * My, ez = sz * kEN + 14.0f * kU * Mz;
    auto row = [&](V4 q) {
        const float ax = fabsf(q.x), ay = fabsf(q.y), az = fabsf(q.z);
        return (ax * ex + ay * ey + az * ez + 10.0f * kU * (ax * (Mx + ex) + ay * (My + ey) + az * (Mz + ez))) * 1.02f;
    };
    const float ecx = row(f.rot0), ecy = row(f.rot1), ecz = row(f.rot2);
    Bounds B;
    B.fx_ecx = fabsf(f.intr.x) * ecx * 1.02f;
    B.fy_ecy = fabsf(f.intr.y) * ecy * 1.02f;
    B.ecz = ecz * kSafe;
    B.kq = (fabsf(a) + 2.0f * fabsf(b) + fabsf(c)) * 1.02f;
    B.gx_ = 2.0f * (fabsf(a) + fabsf(b)) * 1.02f;
    B.gy_ = 2.0f * (fabsf(b) + fabsf(c)) * 1.02f;
    if (!std::isfinite(ecx) || !std::isfinite(ecy) || !std::isfinite(ecz) || !std::isfinite(B.kq))
        B.fx_ecx = B.fy_ecy = B.ecz = B.kq = B.gx_ = B.gy_ = INFINITY;
    return B;
}

// fast_pair: exact draws, approximated radius and angle functions
static bool pair(uint32_t& st, Perturb& pt, float& c, float& s) {
    const float u1 = fmax_(gx::next_u(&st), gxc::kUMin);
    const float u2 = gx::next_u(&st);
    const float le = gx::log(u1);
    const float x = -2.0f * pt.log_(u1);
    const float re = gx::sqrt_(-2.0f * le);
    const float r = fmaxf(re + pt.sgn() * kErMax * kEdge, 0.0f);
    float se, ce;
    gx::sincos(gxc::kTwoPi * u2, &se, &ce);
    c = r * (ce + pt.sgn() * kSinCos * kEdge);
    s = r * (se + pt.sgn() * kSinCos * kEdge);
    return x >= kXMin;
}

// pbvr_fast; R as the renderer's record: r0 (mean xy, depth, o), r1 (keep, eol(o), |fx| ecx,
// |fy| ecy), r2 (centre, a), r3 (b, c, ecz, K), r4 (l00, l10, l11, G_x), r5 (l20, l21, l22, G_y)
static uint32_t fast(const Frame& f, uint32_t W, uint32_t H, uint32_t st, const V4* R, Perturb& pt) {
    float uz, uy, ux, jy;
    bool ok = pair(st, pt, uz, uy);
    ok &= pair(st, pt, ux, jy);
    const V4 r1 = R[1];
    if (f.pbvr[0] == 3u) {
        if (gx::next_u(&st) >= r1.x) return 0u;
    }
    const V4 r2 = R[2], r3 = R[3], r4 = R[4], r5 = R[5];
    const float px = fmaf(r4.x, ux, r2.x) - f.pos.x;
    const float py = fmaf(r4.z, uy, fmaf(r4.y, ux, r2.y)) - f.pos.y;
    const float pz = fmaf(r5.z, uz, fmaf(r5.y, uy, fmaf(r5.x, ux, r2.z))) - f.pos.z;
    const float cz = fmaf(f.rot2.z, pz, fmaf(f.rot2.y, py, f.rot2.x * px));
    const float ecz = r3.z;
    const bool behind = cz + ecz <= f.prm.y;
    const float czl = cz - ecz;
    bool sure = czl > f.prm.y && czl > 3.0f * ecz && cz < 1e30f && czl > 1e-6f;
    const float cx = fmaf(f.rot0.z, pz, fmaf(f.rot0.y, py, f.rot0.x * px));
    const float cy = fmaf(f.rot1.z, pz, fmaf(f.rot1.y, py, f.rot1.x * px));
    const float icz = pt.rcp_(cz);
    const float icl = icz * fmaf((2.0f * kSafe) * ecz, icz, kSafe);
    const float kt = fmaf(ecz, icl, 1e-6f + 2.0f * kU);
    const float tx = (f.intr.x * cx) * icz, ty = (f.intr.y * cy) * icz;
    float pix_x = tx + f.intr.z, pix_y = ty + f.intr.w;
    float epx = fmaf(fabsf(tx), kt, fmaf(r1.z, icl, 2.0f * kU * fabsf(f.intr.z)));
    float epy = fmaf(fabsf(ty), kt, fmaf(r1.w, icl, 2.0f * kU * fabsf(f.intr.w)));
    const uint32_t flags = f.pbvr[2];
    if (flags & 4u) {
        float jx, js;
        sure &= pair(st, pt, jx, js);
        const float sd = gx::sqrt_(fmax_(f.pos.w, 0.0f));
        const float kj = fabsf(sd) * (kEN + 4.0f * kU * kRMax);
        pix_x = pix_x + sd * jx;
        pix_y = pix_y + sd * jy;
        epx = fmaf(4.0f * kU, fabsf(pix_x), epx + kj);
        epy = fmaf(4.0f * kU, fabsf(pix_y), epy + kj);
    }
    sure &= fabsf(pix_x) < 1e30f && fabsf(pix_y) < 1e30f && epx < 1e30f && epy < 1e30f;
    const float mx = kSafe * epx, my = kSafe * epy;
    const bool off = pix_x + mx < 0.0f || pix_x - mx >= (float)W || pix_y + my < 0.0f || pix_y - my >= (float)H;
    uint32_t res = off ? 1u : 2u;
    if (flags & 1u) {
        const V4 r0 = R[0];
        const float dvx = pix_x - r0.x, dvy = pix_y - r0.y;
        const float e = fmaxf(fmaf(2.0f * kU, fabsf(pix_x) + fabsf(r0.x), epx), fmaf(2.0f * kU, fabsf(pix_y) + fabsf(r0.y), epy));
        const float dx2 = dvx * dvx, dy2 = dvy * dvy;
        const float r2v = fmaf(r2.w, dx2, fmaf(2.0f * r3.x, dvx * dvy, r3.y * dy2));
        const float m2 = fmaf(r4.w, dx2, r5.w * dy2);
        const float er2 = fmaf(fmaf(r4.w, fabsf(dvx), r5.w * fabsf(dvy)), e, fmaf(r3.w * e, e, 10.0f * kU * m2));
        const float a2 = fmaxf(r2v, 0.0f);
        const float earg = er2 * (0.5f * kSafe);
        const float oo = fmin_(r0.w, gxc::kOneMinus1e6);
        const float y = oo * pt.exp_(-0.5f * a2);
        const float rel = fmaf(earg, 1.0f + earg, fmaf(0.5f * kExpB, a2, kExpA + 5.4e-7f + 2.0f * kU));
        const float ey = fmaf(y, rel * (1.25f * kSafe), 2.02f * kExpTiny);
        const float v = 1.0f - fmin_(y, gxc::kOneMinus1e6);
        const float ev = ey + 2.0f * kU;
        const float lg = pt.log_(v);
        const float iv = pt.rcp_(v), iy = pt.rcp_(y);
        const float elg = fmaf(kLogRel + 5e-7f, fabsf(lg), kLogAbs + 4e-7f) + ev * iv * fmaf(2.0f * ev, iv, 1.0f) * kSafe;
        const float eo = -lg * iy;
        const float eeo = fmaf(fmaf(fabsf(eo), ey, elg) * iy, fmaf(2.0f * ey, iy, 1.0f) * kSafe, 4e-7f * fabsf(eo));
        sure &= earg < 0.125f && y - ey >= 1e-4f && ev <= 0.5f * v && ey <= 0.5f * y;
        const float de = eeo * kSafe;
        const float ur = gx::next_u(&st) * r1.y;
        const bool reject = ur >= (eo + de) * (1.0f + 6.0f * kU);
        const bool keep = ur * (1.0f + 6.0f * kU) < eo - de;
        res = reject ? 0u : (keep ? res : 2u);
    }
    res = behind ? 0u : (sure ? res : 2u);
    return ok ? res : 2u;
}
}  // namespace fastcheck
}  // namespace o2

// ============================================================================ C entry points
using namespace o2;

static Scene make_scene(const gpsb_gaussian* g, uint32_t n, const float* sh, uint32_t sh_degree, const float* lut) {
    Scene s;
    s.g = g;
    s.n = n;
    s.sh = sh;
    s.sh_max_degree = (sh && sh_degree >= 1 && n > 0) ? std::min(sh_degree, 3u) : 0u;
    uint32_t d = s.sh_max_degree;
    s.sh_stride = d ? (d + 1) * (d + 1) - 1 : 0;
    s.lut = lut;
    double c[3] = {0, 0, 0};
    for (uint32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) c[k] = c[k] + (double)g[i].pos_opacity[k];
    for (int k = 0; k < 3; ++k) s.centroid[k] = n ? c[k] / (double)n : 0.0;
    return s;
}

// Runs fn(begin, end, thread) over [0, n) in chunks taken by `threads` threads in turn.
template <class F>
static void parallel_chunks(uint32_t n, unsigned threads, uint32_t chunk, F fn) {
    if (threads <= 1u) {
        fn(0u, n, 0u);
        return;
    }
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            for (;;) {
                const uint64_t b = next.fetch_add(chunk);
                if (b >= n) break;
                fn((uint32_t)b, (uint32_t)std::min<uint64_t>(n, b + chunk), t);
            }
        });
    for (auto& th : pool) th.join();
}

extern "C" {

// render_ensembles (gps.rs:861-925) for `count` ensembles, in the reference's order.
// accum: W*H*4 floats (in/out). stats: 16 u64 (in/out) in gpsb_stats field order.
// counts_out (nullable): count*n u32 per-splat counts after the cap (0 for the primitive path).
// packed_out (nullable): count*W*H*S u64 packed (depth key << 32 | winner id).
// threads <= 1: the literal sequential form (two passes over the recorded writes). threads > 1:
// every stage split over splats (prepare, particles) or pixels (resolve), each subpixel's winner
// taken by a packed 64-bit minimum; results are identical to the sequential form (tested).
int o2_render_ensembles_mt(const gpsb_gaussian* g, uint32_t n, const float* sh, uint32_t sh_degree,
                           const float* lut, uint32_t W, uint32_t H, uint32_t side,
                           const gpsb_camera* cam, const gpsb_params* prm, uint32_t first_seed, uint32_t count,
                           float* accum, uint64_t* stats, uint32_t* counts_out, uint64_t* packed_out,
                           uint32_t threads) {
    side = std::max(1u, std::min(side, 4u));
    Scene s = make_scene(g, n, sh, sh_degree, lut);
    Stats st;
    memset(&st, 0, sizeof st);
    // stats layout: points, truncated, dropped, visible, orphan, candidates, undercovered, skipped, ensembles,
    // probe, subpixel writes, compact-list entries
    for (int k = 0; k < 12; ++k) st.c[k] = stats[k];
    const uint32_t S = side * side;
    const size_t nsub = (size_t)W * H * S;
    const unsigned T = std::max(1u, threads);
    const bool mt = T > 1u;
    std::vector<uint32_t> depth(mt ? 0 : nsub), winner(mt ? 0 : nsub);
    std::vector<std::atomic<uint64_t>> words(mt ? nsub : 0);
    std::vector<V4> proj((size_t)n * 6u);
    std::vector<uint32_t> offsets(n);
    std::vector<Stats> ts(T);
    bool use_particles = (prm->path == GPSB_PATH_PARTICLE || prm->method != GPSB_METHOD_GPS) && n > 0;
    for (uint32_t e = 0; e < count; ++e) {
        const Frame fr = make_frame(s, *cam, *prm, W, H, side, first_seed + e);
        for (auto& t : ts) memset(&t, 0, sizeof t);
        std::vector<uint64_t> nwrites(T, 0);
        auto pipeline = [&](unsigned t) {
            Pipeline pl(s, mt ? ts[t] : st);
            pl.f = fr;
            pl.W = W; pl.H = H; pl.side = side; pl.S = S;
            pl.proj = proj.data();
            pl.running = 0;
            pl.overflow = false;
            if (mt) pl.packed = words.data();
            return pl;
        };
        std::fill(proj.begin(), proj.end(), V4{0, 0, 0, 0});
        // clear_buffers (gps_splat.wgsl:336-347)
        if (mt) {
            for (auto& w : words) w.store(~0ull, std::memory_order_relaxed);
        } else {
            std::fill(depth.begin(), depth.end(), gxc::kEmpty);
            std::fill(winner.begin(), winner.end(), gxc::kEmpty);
        }
        st.c[8] += 1;
        bool overflow = false;
        std::vector<Write> seq_writes;
        if (use_particles) {
            parallel_chunks(n, T, 4096u, [&](uint32_t b, uint32_t en, unsigned t) {
                Pipeline pl = pipeline(t);
                for (uint32_t i = b; i < en; ++i) offsets[i] = pl.prepare(i);
            });
            if (counts_out) memcpy(counts_out + (size_t)e * n, offsets.data(), (size_t)n * 4);
            uint64_t total = 0;
            for (uint32_t i = 0; i < n; ++i) {
                st.c[11] += offsets[i] ? 1u : 0u;
                total += offsets[i];
            }
            // prepare's exact u32 overflow detection of the running total (gps_splat.wgsl:635-639) and
            // finalize_dispatch (gps_splat.wgsl:648-663): skip the ensemble on u32 overflow
            overflow = total > 0xFFFFFFFFull;
            if (overflow) {
                st.c[7] += 1;
            } else {
                parallel_chunks(n, T, 16u, [&](uint32_t b, uint32_t en, unsigned t) {
                    Pipeline pl = pipeline(t);
                    for (uint32_t i = b; i < en; ++i)
                        for (uint32_t k = 0; k < offsets[i]; ++k) pl.particle(i, k);
                    nwrites[t] += pl.nwrites;
                    if (!mt) seq_writes.swap(pl.writes);
                });
            }
        } else {
            if (counts_out) memset(counts_out + (size_t)e * n, 0, (size_t)n * 4);
            parallel_chunks(n, T, 16u, [&](uint32_t b, uint32_t en, unsigned t) {
                Pipeline pl = pipeline(t);
                for (uint32_t i = b; i < en; ++i) pl.splat_pass(i);
                nwrites[t] += pl.nwrites;
                if (!mt) seq_writes.swap(pl.writes);
            });
        }
        if (mt) {
            for (unsigned t = 0; t < T; ++t) {
                for (int k = 0; k < 16; ++k) st.c[k] += ts[t].c[k];
                st.c[10] += nwrites[t];
                memset(&ts[t], 0, sizeof ts[t]);
            }
        } else {
            st.c[10] += seq_writes.size();
            // depth pass, then colour pass among the depth winners (gps_splat.wgsl:276-281)
            for (const Write& w : seq_writes) depth[w.idx] = std::min(depth[w.idx], w.key);
            for (const Write& w : seq_writes)
                if (depth[w.idx] == w.key) winner[w.idx] = std::min(winner[w.idx], w.id);
        }
        auto word = [&](size_t j) -> uint64_t {
            return mt ? words[j].load(std::memory_order_relaxed) : ((uint64_t)depth[j] << 32) | winner[j];
        };
        if (packed_out) {
            uint64_t* out = packed_out + (size_t)e * nsub;
            for (size_t j = 0; j < nsub; ++j) out[j] = word(j);
        }
        // resolve (gps_splat.wgsl:362-386)
        if (!overflow) {
            parallel_chunks(W * H, T, 4096u, [&](uint32_t b, uint32_t en, unsigned t) {
                Stats& sx = mt ? ts[t] : st;
                for (uint32_t pix = b; pix < en; ++pix) {
                    V3 sum = {(float)0.0, (float)0.0, (float)0.0};
                    for (uint32_t k = 0; k < S; ++k) {
                        const uint64_t w = word((size_t)pix * S + k);
                        const uint32_t dk = (uint32_t)(w >> 32), win = (uint32_t)w;
                        if (dk == gxc::kEmpty) {
                            sum = {sum.x + fr.bg.x, sum.y + fr.bg.y, sum.z + fr.bg.z};
                        } else if (win == gxc::kEmpty) {
                            sx.c[4] += 1;
                            sum = {sum.x + fr.bg.x, sum.y + fr.bg.y, sum.z + fr.bg.z};
                        } else {
                            V3 c = splat_colour(fr, s, win);
                            sum = {sum.x + c.x, sum.y + c.y, sum.z + c.z};
                        }
                    }
                    float* a = accum + (size_t)pix * 4u;
                    a[0] = a[0] + gx::div_(sum.x, (float)S);
                    a[1] = a[1] + gx::div_(sum.y, (float)S);
                    a[2] = a[2] + gx::div_(sum.z, (float)S);
                    a[3] = a[3] + (float)1.0;
                }
            });
            if (mt)
                for (unsigned t = 0; t < T; ++t) st.c[4] += ts[t].c[4];
        }
    }
    for (int k = 0; k < 12; ++k) stats[k] = st.c[k];
    return 0;
}

int o2_render_ensembles(const gpsb_gaussian* g, uint32_t n, const float* sh, uint32_t sh_degree,
                        const float* lut, uint32_t W, uint32_t H, uint32_t side,
                        const gpsb_camera* cam, const gpsb_params* prm, uint32_t first_seed, uint32_t count,
                        float* accum, uint64_t* stats, uint32_t* counts_out, uint64_t* packed_out) {
    return o2_render_ensembles_mt(g, n, sh, sh_degree, lut, W, H, side, cam, prm, first_seed, count, accum, stats,
                                  counts_out, packed_out, 1u);
}

// sp_project + stable radix order + front-to-back f32 blend (the sorted path; see the file
// header for the blend arithmetic). keys/vals: n u32 each (sorted output). accum: overwritten
// with (rgb, 1). stats[9] (probe_demand) is overwritten with the GPS demand of the view.
int o2_render_sorted(const gpsb_gaussian* g, uint32_t n, const float* sh, uint32_t sh_degree,
                     const float* lut, uint32_t W, uint32_t H, uint32_t side,
                     const gpsb_camera* cam, const gpsb_params* prm_in,
                     float* accum, uint64_t* stats, uint32_t* keys_out, uint32_t* vals_out) {
    side = std::max(1u, std::min(side, 4u));
    gpsb_params prm = *prm_in;
    prm.method = GPSB_METHOD_GPS;
    Scene s = make_scene(g, n, sh, sh_degree, lut);
    Stats st;
    memset(&st, 0, sizeof st);
    Pipeline pl(s, st);
    pl.f = make_frame(s, *cam, prm, W, H, side, 0u);
    pl.W = W; pl.H = H; pl.side = side; pl.S = side * side;
    struct Rec { float mx, my, o, K, w1x, w1y, w2x, w2y; V3 col; };
    std::vector<Rec> rec(n);
    std::vector<uint32_t> keys(n), vals(n);
    uint64_t demand = 0;
    for (uint32_t i = 0; i < n; ++i) {
        // sp_project (gps_splat.wgsl:737-777)
        keys[i] = 0xFFFFFFu;
        vals[i] = i;
        Proj pr = project(pl.f, g[i]);
        if (!pr.ok) continue;
        float o = gx::clamp_(g[i].pos_opacity[3], (float)0.0, (float)1.0);
        if (o <= (float)0.0 || pl.offscreen(pr)) continue;
        float en = pl.expected_count(pr, o);
        if (en > (float)0.0) demand += gx::f2u(fmin_(en, (float)4.0e9));
        if (o < gxc::kSpMinAlpha) continue;
        float K = gx::sqrt_((float)2.0 * gx::log(gx::div_(o, gxc::kSpMinAlpha)));
        float ex = K * gx::sqrt_(pr.a), ey = K * gx::sqrt_(pr.c);
        if (pr.mx + ex < (float)0.0 || pr.mx - ex >= (float)W || pr.my + ey < (float)0.0 || pr.my - ey >= (float)H) continue;
        float tr2 = (float)0.5 * (pr.a + pr.c);
        float disc = gx::sqrt_(fmax_(tr2 * tr2 - (pr.a * pr.c - pr.b * pr.b), (float)0.0));
        float l1 = tr2 + disc;
        float l2 = fmax_(tr2 - disc, (float)1e-12);
        float v1x = (float)1.0, v1y = (float)0.0;
        if (fabsf(pr.b) > (float)1e-12) {
            float ux = l1 - pr.c, uy = pr.b;
            float len = gx::sqrt_(ux * ux + uy * uy);
            v1x = gx::div_(ux, len);
            v1y = gx::div_(uy, len);
        } else if (pr.a < pr.c) {
            v1x = (float)0.0;
            v1y = (float)1.0;
        }
        float v2x = -v1y, v2y = v1x;
        float s1 = gx::sqrt_(l1), s2 = gx::sqrt_(l2);
        rec[i] = {pr.mx, pr.my, o, K, gx::div_(v1x, s1), gx::div_(v1y, s1), gx::div_(v2x, s2), gx::div_(v2y, s2),
                  splat_colour(pl.f, s, i)};
        keys[i] = 0xFFFFFEu - (gx::f2b(pr.depth) >> 8u);
    }
    // stable ascending sort of (key, id) = the LSD radix result (gps_sort.wgsl:1-50)
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    uint32_t valid = 0;
    for (uint32_t j = 0; j < n; ++j) {
        keys_out[j] = keys[order[j]];
        vals_out[j] = vals[order[j]];
        if (keys_out[j] != 0xFFFFFFu) valid = j + 1;
    }
    // front-to-back blend of the valid entries, nearest (last) first
    for (uint32_t y = 0; y < H; ++y)
        for (uint32_t x = 0; x < W; ++x) {
            float pcx = (float)x + (float)0.5, pcy = (float)y + (float)0.5;
            float T = (float)1.0, cr = (float)0.0, cgr = (float)0.0, cb = (float)0.0;
            for (uint32_t j = valid; j-- > 0;) {
                const Rec& r = rec[vals_out[j]];
                float dx = pcx - r.mx, dy = pcy - r.my;
                float u = dx * r.w1x + dy * r.w1y;
                float v = dx * r.w2x + dy * r.w2y;
                float r2 = u * u + v * v;
                if (r2 > r.K * r.K) continue;
                float alpha = fmin_(r.o * gx::exp(-(float)0.5 * r2), (float)0.99);
                if (alpha < gxc::kSpMinAlpha) continue;
                float wgt = T * alpha;
                cr = cr + wgt * r.col.x;
                cgr = cgr + wgt * r.col.y;
                cb = cb + wgt * r.col.z;
                T = T * ((float)1.0 - alpha);
                if (T < (float)1e-4) break;
            }
            float* a = accum + ((size_t)y * W + x) * 4u;
            a[0] = cr + T * prm.background[0];
            a[1] = cgr + T * prm.background[1];
            a[2] = cb + T * prm.background[2];
            a[3] = (float)1.0;
        }
    stats[9] = demand;
    return 0;
}

static float oetf(float c) {
    if (c <= (float)0.0031308) return (float)12.92 * c;
    return (float)1.055 * gx::pow(c, gxc::kInv2p4) - (float)0.055;
}

// gps_composite.wgsl:41-55 into an RGBA8 buffer of out_w x out_h.
int o2_composite(const float* accum, uint32_t W, uint32_t H, float exposure, uint32_t gamma_on,
                 uint32_t out_w, uint32_t out_h, uint8_t* out) {
    auto lin = [&](int px, int py, float* c) {
        int qx = std::min(std::max(px, 0), (int)W - 1), qy = std::min(std::max(py, 0), (int)H - 1);
        const float* a = accum + ((size_t)qy * W + qx) * 4u;
        float d = fmax_(a[3], (float)1.0);
        c[0] = gx::div_(a[0], d);
        c[1] = gx::div_(a[1], d);
        c[2] = gx::div_(a[2], d);
    };
    for (uint32_t Y = 0; Y < out_h; ++Y)
        for (uint32_t X = 0; X < out_w; ++X) {
            float uvx = gx::div_((float)X + (float)0.5, (float)out_w), uvy = gx::div_((float)Y + (float)0.5, (float)out_h);
            float qx = uvx * (float)W - (float)0.5, qy = uvy * (float)H - (float)0.5;
            float fx0 = floorf(qx), fy0 = floorf(qy);
            int px = (int)fx0, py = (int)fy0;
            float fx = qx - fx0, fy = qy - fy0;
            float c00[3], c10[3], c01[3], c11[3];
            lin(px, py, c00); lin(px + 1, py, c10); lin(px, py + 1, c01); lin(px + 1, py + 1, c11);
            uint8_t* o = out + ((size_t)Y * out_w + X) * 4u;
            for (int k = 0; k < 3; ++k) {
                float top = mix(c00[k], c10[k], fx), bot = mix(c01[k], c11[k], fx);
                float c = mix(top, bot, fy) * exposure;
                c = gx::clamp_(c, (float)0.0, (float)1.0);
                if (gamma_on) c = oetf(c);
                o[k] = (uint8_t)gx::f2u(gx::rint_(c * (float)255.0));
            }
            o[3] = 255;
        }
    return 0;
}

// Shared-function probes for the fmath tests: out[i] = f(in[i]) for f in {exp, log, sin, cos}.
// The fast-decision check (fastcheck above) over every particle of `count` ensembles of a PBVR
// frame: out[0] particles, out[1] decided by the restated fast path, out[2] decided wrongly,
// out[3] points among the particles. mode: 0 random perturbation signs (seeded by perturb_seed),
// 1 all +, 2 all -.
int o2_fast_check(const gpsb_gaussian* g, uint32_t n, const float* sh, uint32_t sh_degree, const float* lut,
                  uint32_t W, uint32_t H, uint32_t side, const gpsb_camera* cam, const gpsb_params* prm,
                  uint32_t first_seed, uint32_t count, uint32_t perturb_seed, int mode, uint64_t* out) {
    side = std::max(1u, std::min(side, 4u));
    if (prm->method == GPSB_METHOD_GPS || prm->method == GPSB_METHOD_SCREEN_OCCUPANCY) return -1;
    Scene s = make_scene(g, n, sh, sh_degree, lut);
    Stats st;
    memset(&st, 0, sizeof st);
    fastcheck::Perturb pt{perturb_seed * 2654435761u + 1u, mode};
    for (int k = 0; k < 4; ++k) out[k] = 0;
    for (uint32_t e = 0; e < count; ++e) {
        Pipeline pl(s, st);
        pl.f = make_frame(s, *cam, *prm, W, H, side, first_seed + e);
        pl.W = W; pl.H = H; pl.side = side; pl.S = side * side;
        std::vector<V4> proj((size_t)n * 6u, V4{0, 0, 0, 0});
        pl.proj = proj.data();
        pl.running = 0;
        pl.overflow = false;
        std::vector<uint32_t> cnt(n);
        for (uint32_t i = 0; i < n; ++i) cnt[i] = pl.prepare(i);
        if (pl.overflow) continue;
        for (uint32_t i = 0; i < n; ++i) {
            if (!cnt[i]) continue;
            const V4* P = &pl.proj[(size_t)i * 6u];
            const V4 a = P[0], b = P[1], c = P[2], d = P[3], e4 = P[4], f4 = P[5];
            const V3 ca = {e4.x, e4.y, e4.z}, cb = {f4.x, f4.y, f4.z};
            const fastcheck::Bounds B = fastcheck::bounds_of(pl.f, {c.x, c.y, c.z}, ca, cb, c.w, d.x, d.y);
            const float h = Pipeline::eol(fmin_(a.w, gxc::kOneMinus1e6));
            const V4 R[6] = {a, {b.w, h, B.fx_ecx, B.fy_ecy}, c, {d.x, d.y, B.ecz, B.kq},
                             {ca.x, ca.y, ca.z, B.gx_}, {cb.x, cb.y, cb.z, B.gy_}};
            for (uint32_t k = 0; k < cnt[i]; ++k) {
                const uint32_t seed = gx::particle_seed(i, k + 1u, pl.f.cfg[0]);
                Rng rng{seed, false, (float)0.0};
                uint32_t idx;
                float dz;
                const uint32_t exact = pl.pbvr_eval(rng, a, b, c, d, ca, cb, idx, dz);
                const uint32_t q = fastcheck::fast(pl.f, W, H, seed, R, pt);
                out[0] += 1;
                out[3] += exact & 1u;
                if (q != 2u) {
                    out[1] += 1;
                    out[2] += q != exact ? 1u : 0u;
                }
            }
        }
    }
    return 0;
}

void o2_fmath_eval(int which, const float* in, float* out, size_t n) {
    for (size_t i = 0; i < n; ++i) {
        float x = in[i];
        out[i] = which == 0 ? gx::exp(x) : which == 1 ? gx::log(x) : which == 2 ? gx::sin(x) : which == 3 ? gx::cos(x)
                 : which == 5 ? gx::log_t_pos(x, gx::tab_log()) : gx::pow(x, gxc::kInv2p4);
    }
}

}  // extern "C"
