// O1: f64 semantic oracle, a C++ restatement of crates/gps-core (lib.rs, oracle.rs, camera.rs).
// TEST INFRASTRUCTURE AND CPU BASELINE ONLY: the product renderer never calls this file.
//
// The reference's own arithmetic dependency, glam 0.29.3 (Cargo.lock; not vendored in the
// reference), is restated by the small column-major Vec/Mat helpers below: DMat3::from_quat,
// DMat2::inverse/determinant, DQuat::normalize and the matrix products used at
// crates/gps-core/src/lib.rs:94-105 and oracle.rs:116-136, 352-418. It is pinned the same way the
// reference pins it: by the six golden images of the original C++ oracle
// (tests/fixtures/cpp_*.f64, thresholds of crates/gps-core/tests/cpp_crosscheck.rs:57-100) and by
// the analytic vectors of crates/gps-core/src/vectors.rs.
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <vector>
#include <algorithm>
#include <thread>
#include <atomic>

namespace o1 {

static const double PI = 3.14159265358979323846;
static const double SH_C0 = 0.28209479177387814;     // lib.rs:15
static const double DILOG_AT_ONE = 1.6449340668482264; // lib.rs:17

struct V2 { double x, y; };
struct V3 { double x, y, z; };
static inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 mul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
static inline double length(V3 a) { return sqrt(dot(a, a)); }
static inline V3 normalize(V3 a) { return mul(a, 1.0 / length(a)); }

// column-major 3x3 (glam DMat3): c[col].{x,y,z}
struct M3 { V3 c[3]; };
static inline V3 mv(const M3& m, V3 v) { return add(add(mul(m.c[0], v.x), mul(m.c[1], v.y)), mul(m.c[2], v.z)); }
static inline M3 mm(const M3& a, const M3& b) { return {{mv(a, b.c[0]), mv(a, b.c[1]), mv(a, b.c[2])}}; }
static inline M3 transpose(const M3& m) {
    return {{{m.c[0].x, m.c[1].x, m.c[2].x}, {m.c[0].y, m.c[1].y, m.c[2].y}, {m.c[0].z, m.c[1].z, m.c[2].z}}};
}
static inline M3 from_rows(const double* r) {  // row-major 9 -> column-major
    return {{{r[0], r[3], r[6]}, {r[1], r[4], r[7]}, {r[2], r[5], r[8]}}};
}
// column-major 2x2 (glam DMat2): x = column 0, y = column 1
struct M2 { V2 x, y; };
static inline double det2(const M2& m) { return m.x.x * m.y.y - m.y.x * m.x.y; }
static inline M2 inverse2(const M2& m) {
    double inv = 1.0 / det2(m);
    return {{m.y.y * inv, m.x.y * -inv}, {m.y.x * -inv, m.x.x * inv}};
}
static inline V2 mv2(const M2& m, V2 v) { return {m.x.x * v.x + m.y.x * v.y, m.x.y * v.x + m.y.y * v.y}; }

struct Quat { double x, y, z, w; };
static inline Quat qnormalize(Quat q) {
    double len = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    double r = 1.0 / len;
    return {q.x * r, q.y * r, q.z * r, q.w * r};
}
// DMat3::from_quat (unit quaternion -> rotation), the standard formula.
static M3 from_quat(Quat q) {
    double x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
    double xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
    double yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
    double wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
    return {{{1.0 - (yy + zz), xy + wz, xz - wy}, {xy - wz, 1.0 - (xx + zz), yz + wx}, {xz + wy, yz - wx, 1.0 - (xx + yy)}}};
}

// ------------------------------------------------------------------ lib.rs
double sigmoid(double x) { return 1.0 / (1.0 + exp(-x)); }  // lib.rs:21-23
static inline int sh_rest_per_channel(int d) { return (d + 1) * (d + 1) - 1; }

// eval_sh (lib.rs:36-87)
V3 eval_sh(int degree, V3 dc, const double* rest, V3 dir, int stride) {
    const double C1 = 0.4886025119029199;
    const double C2[5] = {1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396};
    const double C3[7] = {-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154,
                          -0.4570457994644658, 1.445305721320277, -0.5900435899266435};
    V3 res = mul(dc, SH_C0);
    degree = std::min(degree, 3);
    if (degree >= 1 && rest) {
        int r = std::max(stride, sh_rest_per_channel(degree));
        auto sh = [&](int k) { return V3{rest[k], rest[r + k], rest[2 * r + k]}; };
        double x = dir.x, y = dir.y, z = dir.z;
        res = add(res, sub(add(mul(sh(0), -C1 * y), mul(sh(1), C1 * z)), mul(sh(2), C1 * x)));
        if (degree >= 2) {
            double xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            V3 t = add(add(add(add(mul(sh(3), C2[0] * xy), mul(sh(4), C2[1] * yz)), mul(sh(5), C2[2] * (2.0 * zz - xx - yy))),
                           mul(sh(6), C2[3] * xz)), mul(sh(7), C2[4] * (xx - yy)));
            res = add(res, t);
            if (degree >= 3) {
                V3 u = add(add(add(add(add(add(mul(sh(8), C3[0] * y * (3.0 * xx - yy)), mul(sh(9), C3[1] * xy * z)),
                                           mul(sh(10), C3[2] * y * (4.0 * zz - xx - yy))),
                                       mul(sh(11), C3[3] * z * (2.0 * zz - 3.0 * xx - 3.0 * yy))),
                                   mul(sh(12), C3[4] * x * (4.0 * zz - xx - yy))),
                               mul(sh(13), C3[5] * z * (xx - yy))),
                           mul(sh(14), C3[6] * x * (xx - 3.0 * yy)));
                res = add(res, u);
            }
        }
    }
    res = add(res, V3{0.5, 0.5, 0.5});
    return {std::max(res.x, 0.0), std::max(res.y, 0.0), std::max(res.z, 0.0)};
}

M3 covariance_3d(V3 log_scale, Quat rot) {  // lib.rs:98-106
    M3 r = from_quat(qnormalize(rot));
    M3 s2 = {{{exp(2.0 * log_scale.x), 0, 0}, {0, exp(2.0 * log_scale.y), 0}, {0, 0, exp(2.0 * log_scale.z)}}};
    return mm(mm(r, s2), transpose(r));
}

struct Pinhole { M3 view_rot; V3 view_pos; double fx, fy, tan_fov_x, tan_fov_y; };
static inline V3 world_to_camera(const Pinhole& c, V3 w) { return mv(c.view_rot, sub(w, c.view_pos)); }

M2 covariance_2d(const M3& cov3d, V3 mean_world, const Pinhole& cam, double low_pass) {  // lib.rs:137-165
    V3 t = world_to_camera(cam, mean_world);
    double limx = 1.3 * cam.tan_fov_x, limy = 1.3 * cam.tan_fov_y;
    double txtz = t.x / t.z, tytz = t.y / t.z;
    t.x = std::min(std::max(txtz, -limx), limx) * t.z;
    t.y = std::min(std::max(tytz, -limy), limy) * t.z;
    M3 j = {{{cam.fx / t.z, 0.0, 0.0}, {0.0, cam.fy / t.z, 0.0},
             {-cam.fx * t.x / (t.z * t.z), -cam.fy * t.y / (t.z * t.z), 0.0}}};
    M3 tm = mm(j, cam.view_rot);
    M3 cov = mm(mm(tm, cov3d), transpose(tm));
    M2 c2 = {{cov.c[0].x, cov.c[0].y}, {cov.c[1].x, cov.c[1].y}};
    c2.x.x += low_pass;
    c2.y.y += low_pass;
    return c2;
}

M2 cholesky_2d(const M2& a) {  // lib.rs:168-174
    double eps = 1e-300;
    double l00 = sqrt(std::max(a.x.x, eps));
    double l10 = a.x.y / l00;
    double l11 = sqrt(std::max(a.y.y - l10 * l10, eps));
    return {{l00, l10}, {0.0, l11}};
}

static double dilog_series(double x) {  // lib.rs:178-190
    double term = x, sum = x;
    for (int k = 2; k < 1000; ++k) {
        term *= x;
        double add = term / ((double)k * (double)k);
        sum += add;
        if (fabs(add) < 1e-18 * fabs(sum)) break;
    }
    return sum;
}
double dilog(double x) {  // lib.rs:193-212
    if (x >= 1.0) return DILOG_AT_ONE;
    if (x <= -1.0) return -DILOG_AT_ONE / 2.0;
    if (x == 0.0) return 0.0;
    if (x < 0.0) {
        double y = x / (x - 1.0);
        double l = log(1.0 - x);
        return -dilog_series(y) - 0.5 * l * l;
    }
    if (x <= 0.5) return dilog_series(x);
    return DILOG_AT_ONE - log(x) * log(1.0 - x) - dilog_series(1.0 - x);
}
double inv_dilog(double target) {  // lib.rs:219-248
    double top;
    uint64_t b;
    memcpy(&b, &DILOG_AT_ONE, 8);
    b -= 1;
    memcpy(&top, &b, 8);
    target = std::min(std::max(target, 0.0), top);
    if (target <= 0.0) return 0.0;
    double lo = 0.0, hi = 1.0, y = target / DILOG_AT_ONE;
    for (int it = 0; it < 40; ++it) {
        double f = dilog(y) - target;
        if (f > 0.0) hi = y; else lo = y;
        double dfdy = (y > 1e-12 && y < 1.0 - 1e-15) ? -log(1.0 - y) / y : 1.0;
        double ny = y - f / dfdy;
        if (!(ny > lo && ny < hi)) ny = 0.5 * (lo + hi);
        if (fabs(ny - y) <= 1e-14 * (1.0 + y)) return ny;
        y = ny;
    }
    return y;
}
double expected_point_count(double det, double o) {  // lib.rs:253-258
    if (det <= 0.0 || o <= 0.0) return 0.0;
    return 2.0 * PI * sqrt(det) * dilog(std::min(o, 1.0));
}
double pixel_density_scale(double depth, double fx, double fy, double refl, double near_z) {  // lib.rs:260-280
    if (!std::isfinite(depth) || !std::isfinite(fx) || !std::isfinite(fy) || !std::isfinite(refl) || !std::isfinite(near_z) ||
        depth <= std::max(near_z, 0.0) || fx <= 0.0 || fy <= 0.0 || refl <= 0.0)
        return 0.0;
    double ratio = refl / depth;
    return std::min(ratio * ratio * fx * fy, 1.0e12);
}
static const double MAX_OPACITY = 1.0 - 1e-12;
double projected_footprint_area(const M2& c) {  // lib.rs:287-293
    double det = c.x.x * c.y.y - c.y.x * c.x.y;
    if (!std::isfinite(det) || det <= 0.0) return 0.0;
    return 2.0 * PI * sqrt(det);
}
enum Rule { PROPORTIONAL = 0, EXTINCTION = 1, DILOG = 2 };
double opacity_term(int rule, double o) {  // lib.rs:302-312
    if (!std::isfinite(o) || o <= 0.0) return 0.0;
    o = std::min(o, MAX_OPACITY);
    if (rule == PROPORTIONAL) return o;
    if (rule == EXTINCTION) return -log1p(-o);
    return dilog(o);
}
struct CalIn { double object_depth, splat_depth, fx, fy, near_z, refl, footprint_area, spp; };
double calibrated_count(int level, int rule, double o, double base_k, double density, const CalIn& in) {  // lib.rs:349-391
    double g = opacity_term(rule, o);
    if (!(g > 0.0) || !std::isfinite(density) || density <= 0.0) return 0.0;
    double scale;
    if (level == 0) scale = base_k;
    else if (level == 1) scale = base_k * pixel_density_scale(in.object_depth, in.fx, in.fy, in.refl, in.near_z);
    else if (level == 2) scale = base_k * pixel_density_scale(in.splat_depth, in.fx, in.fy, in.refl, in.near_z);
    else scale = in.spp * in.footprint_area;
    double n = density * g * scale;
    return (std::isfinite(n) && n > 0.0) ? n : 0.0;
}
static double extinction_over_linear(double x) { return x < 1e-8 ? 1.0 + 0.5 * x : -log1p(-x) / x; }  // lib.rs:393-399
double radial_keep_probability(double o, double r2) {  // lib.rs:402-410
    if (!std::isfinite(o) || o <= 0.0) return 1.0;
    if (std::isnan(r2) || r2 < 0.0) r2 = 0.0;
    o = std::min(o, MAX_OPACITY);
    double y = o * exp(-0.5 * r2);
    return std::min(std::max(extinction_over_linear(y) / extinction_over_linear(o), 0.0), 1.0);
}
double footprint_point_count(double expected, uint32_t s) {  // lib.rs:412-418
    if (!std::isfinite(expected) || expected <= 0.0) return 0.0;
    double ss = (double)std::max(s, 1u);
    return expected / (ss * ss);
}
uint32_t adaptive_footprint(double sigma_min, double kappa, uint32_t s_max) {  // lib.rs:420-433
    if (!(kappa > 0.0) || !std::isfinite(sigma_min) || sigma_min <= 0.0) return 1;
    uint32_t hi = std::max(s_max, 1u);
    double s = floor(kappa * sigma_min);
    if (!(s >= 1.0)) return 1;
    if (s >= (double)hi) return hi;
    return (uint32_t)s;
}
uint32_t pcg_hash(uint32_t v) {  // lib.rs:438-442
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
uint32_t particle_seed(bool frame_varying, uint32_t splat, uint32_t k, uint32_t frame) {  // lib.rs:450-465
    uint32_t s = pcg_hash(splat * 747796405u + k + 1u);
    if (frame_varying) s = pcg_hash(s ^ (frame * 2654435761u + 1u));
    return s ? s : 1u;
}
struct RandStream {  // lib.rs:469-498
    uint32_t state;
    bool has_spare;
    double spare;
    explicit RandStream(uint32_t seed) : state(seed ? seed : 0x9E3779B9u), has_spare(false), spare(0) {}
    double next() {
        state = pcg_hash(state);
        return (double)state * (1.0 / 4294967296.0);
    }
    double normal() {
        if (has_spare) { has_spare = false; return spare; }
        double u1 = std::max(next(), 1e-300);
        double u2 = next();
        double r = sqrt(-2.0 * log(u1));
        double th = 2.0 * PI * u2;
        spare = r * sin(th);
        has_spare = true;
        return r * cos(th);
    }
};
int32_t poisson_sample(double lambda, RandStream& rng) {  // lib.rs:500-519
    if (lambda <= 0.0) return 0;
    if (lambda < 30.0) {
        double l = exp(-lambda);
        int32_t k = 0;
        double p = 1.0;
        for (;;) {
            k += 1;
            p *= rng.next();
            if (p <= l) break;
        }
        return k - 1;
    }
    double n = round(lambda + sqrt(lambda) * rng.normal());
    n = std::max(n, 0.0);
    return n >= 2147483647.0 ? 2147483647 : (int32_t)n;
}
double sample_corrected_radius(double opacity, double u) {  // lib.rs:522-536
    double o = std::min(std::max(opacity, 0.0), 1.0);
    if (o <= 0.0) return 0.0;
    u = std::min(std::max(u, 0.0), 1.0);
    double d = dilog(o);
    double target = (1.0 - u) * d;
    double y = std::min(inv_dilog(target), o);
    if (y <= 0.0) return 40.0;
    double r2 = -2.0 * log(y / o);
    return sqrt(std::max(r2, 0.0));
}
V2 sample_corrected_offset(double opacity, const M2& cov, RandStream& rng) {  // lib.rs:538-542
    double r = sample_corrected_radius(opacity, rng.next());
    double th = 2.0 * PI * rng.next();
    return mv2(cholesky_2d(cov), V2{r * cos(th), r * sin(th)});
}

struct Gaussian2D { V2 mean; M2 cov; double opacity; V3 color; double depth; };
double alpha_at(const Gaussian2D& g, V2 p) {  // lib.rs:555-559
    V2 d = {p.x - g.mean.x, p.y - g.mean.y};
    V2 id = mv2(inverse2(g.cov), d);
    double m = d.x * id.x + d.y * id.y;
    return std::min(std::max(g.opacity, 0.0), 1.0) * exp(-0.5 * m);
}
double expected_coverage(double a, double area) {  // lib.rs:561-564
    a = std::min(std::max(a, 0.0), 1.0 - 1e-15);
    return 1.0 - pow(1.0 - a, area);
}
V3 composite_expected(const std::vector<Gaussian2D>& sorted_layers, V2 p, V3 bg, double area) {  // lib.rs:567-585
    V3 acc = {0, 0, 0};
    double t = 1.0;
    for (const auto& g : sorted_layers) {
        double a = expected_coverage(alpha_at(g, p), area);
        acc = add(acc, mul(g.color, t * a));
        t *= 1.0 - a;
        if (t <= 1e-9) break;
    }
    return add(acc, mul(bg, t));
}
uint32_t ordered_depth_key(float depth) {  // lib.rs:590-594
    uint32_t b;
    memcpy(&b, &depth, 4);
    return b ^ ((b & 0x80000000u) ? 0xFFFFFFFFu : 0x80000000u);
}
float ordered_depth_key_inverse(uint32_t key) {  // lib.rs:596-599
    uint32_t b = key ^ ((key & 0x80000000u) ? 0x80000000u : 0xFFFFFFFFu);
    float f;
    memcpy(&f, &b, 4);
    return f;
}
// radius_lut (lib.rs:624-636)
void radius_lut(float* t) {
    const int NO = 65, NV = 129;
    const double VMAX = 17.0;
    for (int i = 0; i < NO; ++i) {
        double x = (double)i / (double)(NO - 1);
        double o = std::min(std::max(1.0 - (1.0 - x) * (1.0 - x), 1e-6), 1.0);
        for (int j = 0; j < NV; ++j) {
            double w = (double)j * sqrt(VMAX) / (double)(NV - 1);
            double u = -expm1(-w * w);
            t[i * NV + j] = (float)sample_corrected_radius(o, u);
        }
    }
}
// radius_from_lut (lib.rs:639-648)
double radius_from_lut(const float* lut, double o, double u) {
    double v = -log(std::max(1.0 - u, 6e-8));
    double fo = (1.0 - sqrt(1.0 - std::min(std::max(o, 0.0), 1.0))) * 64.0;
    double fv = std::min(std::max(sqrt(v) / sqrt(17.0), 0.0), 1.0) * 128.0;
    size_t i0 = std::min((size_t)fo, (size_t)63), j0 = std::min((size_t)fv, (size_t)127);
    double a = fo - (double)i0, b = fv - (double)j0;
    auto at = [&](size_t i, size_t j) { return (double)lut[i * 129 + j]; };
    double r = (1.0 - a) * ((1.0 - b) * at(i0, j0) + b * at(i0, j0 + 1)) + a * ((1.0 - b) * at(i0 + 1, j0) + b * at(i0 + 1, j0 + 1));
    return std::max(r, 0.0);
}

// ------------------------------------------------------------------ oracle.rs
struct Gaussian3D { V3 pos; V3 log_scale; Quat rot; double opacity; V3 color; };
struct Camera { M3 view_rot; V3 view_pos; double fx, fy, cx, cy, low_pass; };

static Pinhole to_pinhole(const Camera& c) { return {c.view_rot, c.view_pos, c.fx, c.fy, 4.0, 4.0}; }  // oracle.rs:72-82
static Camera with_default_pp(Camera c, size_t w, size_t h) {  // oracle.rs:84-90
    if (c.cx == 0.0 && c.cy == 0.0) { c.cx = 0.5 * (double)w; c.cy = 0.5 * (double)h; }
    return c;
}
struct Projected { V2 mean; M2 cov2d; double det, depth, opacity; V3 color; };
static bool project(const Gaussian3D& g, const Camera& c, Projected& out) {  // oracle.rs:116-136
    Pinhole pin = to_pinhole(c);
    V3 cm = world_to_camera(pin, g.pos);
    if (cm.z <= 1e-4) return false;
    M3 c3 = covariance_3d(g.log_scale, g.rot);
    M2 c2 = covariance_2d(c3, g.pos, pin, c.low_pass);
    double det = det2(c2);
    if (det <= 0.0) return false;
    out.mean = {c.fx * cm.x / cm.z + c.cx, c.fy * cm.y / cm.z + c.cy};
    out.cov2d = c2;
    out.det = det;
    out.depth = cm.z;
    out.opacity = std::min(std::max(g.opacity, 0.0), 1.0);
    out.color = g.color;
    return true;
}
struct RenderStats { double points, candidates, subpixel_writes; };

static inline void depth_test(size_t idx, double d, V3 c, double* depth, V3* color, RenderStats& st) {  // oracle.rs:147-153
    st.subpixel_writes += 1.0;
    if (d < depth[idx]) { depth[idx] = d; color[idx] = c; }
}
static void write_block(V2 pixel, int64_t s, size_t w, size_t h, int64_t side, double d, V3 c, double* depth, V3* color,
                        RenderStats& st) {  // oracle.rs:156-173
    int64_t spp = side * side;
    int64_t gx0 = (int64_t)floor(pixel.x * (double)side - 0.5 * (double)s + 0.5);
    int64_t gy0 = (int64_t)floor(pixel.y * (double)side - 0.5 * (double)s + 0.5);
    int64_t gw = (int64_t)w * side, gh = (int64_t)h * side;
    for (int64_t gy = std::max(gy0, (int64_t)0); gy < std::min(gh, gy0 + s); ++gy)
        for (int64_t gx = std::max(gx0, (int64_t)0); gx < std::min(gw, gx0 + s); ++gx) {
            int64_t px = gx / side, py = gy / side, sx = gx % side, sy = gy % side;
            size_t idx = (size_t)(((int64_t)((size_t)py * w + (size_t)px)) * spp + sy * side + sx);
            depth_test(idx, d, c, depth, color, st);
        }
}
static void resolve_set(size_t w, size_t h, size_t spp, const double* depth, const V3* color, V3 bg, V3* accum) {  // oracle.rs:175-186
    for (size_t y = 0; y < h; ++y)
        for (size_t x = 0; x < w; ++x) {
            size_t base = (y * w + x) * spp;
            V3 sum = {0, 0, 0};
            for (size_t k = 0; k < spp; ++k) sum = add(sum, depth[base + k] < 1e299 ? color[base + k] : bg);
            accum[y * w + x] = add(accum[y * w + x], mul(sum, 1.0 / (double)spp));
        }
}

void render_analytic(const Gaussian3D* scene, size_t n, Camera cam, size_t w, size_t h, V3 bg, V3* img) {  // oracle.rs:190-200
    cam = with_default_pp(cam, w, h);
    std::vector<Gaussian2D> layers;
    for (size_t i = 0; i < n; ++i) {
        Projected p;
        if (project(scene[i], cam, p)) layers.push_back({p.mean, p.cov2d, p.opacity, p.color, p.depth});
    }
    std::stable_sort(layers.begin(), layers.end(), [](const Gaussian2D& a, const Gaussian2D& b) { return a.depth < b.depth; });
    for (size_t y = 0; y < h; ++y)
        for (size_t x = 0; x < w; ++x) img[y * w + x] = composite_expected(layers, V2{x + 0.5, y + 0.5}, bg, 1.0);
}

struct MCOptions {  // oracle.rs:205-226
    uint32_t footprint_subpixels;
    double adaptive_kappa;
    uint32_t footprint_max;
    int compensate_blur;
    double density_scale;
    int per_particle_seed;
    uint32_t max_points_per_splat;
};
static const double OFFSCREEN_SIGMA = 5.9;

// render_monte_carlo (oracle.rs:229-312). Sets [set_lo, set_hi) only, accumulated without the
// final division (so ensembles can be split across threads and summed in set order).
static void mc_sets(const std::vector<Projected>& proj, const std::vector<uint32_t>& footprint, const std::vector<M2>& sample_cov,
                    size_t w, size_t h, size_t side, V3 bg, uint32_t base_seed, const MCOptions& opt, size_t set_lo,
                    size_t set_hi, V3* accum, RenderStats& st) {
    size_t spp = side * side, n_sub = w * h * spp;
    std::vector<double> depth(n_sub);
    std::vector<V3> color(n_sub);
    for (size_t s = set_lo; s < set_hi; ++s) {
        std::fill(depth.begin(), depth.end(), 1e300);
        std::fill(color.begin(), color.end(), V3{0, 0, 0});
        for (size_t gid = 0; gid < proj.size(); ++gid) {
            const Projected& pr = proj[gid];
            uint32_t fp = footprint[gid];
            double en = footprint_point_count(expected_point_count(pr.det, pr.opacity) * (double)spp * opt.density_scale, fp);
            if (en <= 0.0) continue;
            if (fp == 1) {
                double ex = OFFSCREEN_SIGMA * sqrt(sample_cov[gid].x.x), ey = OFFSCREEN_SIGMA * sqrt(sample_cov[gid].y.y);
                if (pr.mean.x + ex < 0.0 || pr.mean.x - ex >= (double)w || pr.mean.y + ey < 0.0 || pr.mean.y - ey >= (double)h) continue;
            }
            uint32_t frame = base_seed + (uint32_t)s;
            RandStream rng(particle_seed(true, (uint32_t)gid, 0, frame));
            int32_t n_full = poisson_sample(en, rng);
            st.points += (double)n_full;
            int32_t n = (int32_t)std::min((uint32_t)n_full, opt.max_points_per_splat);
            for (int32_t j = 0; j < n; ++j) {
                if (opt.per_particle_seed) rng = RandStream(particle_seed(true, (uint32_t)gid, (uint32_t)j + 1u, frame));
                V2 off = sample_corrected_offset(pr.opacity, sample_cov[gid], rng);
                V2 pixel = {pr.mean.x + off.x, pr.mean.y + off.y};
                if (fp == 1) {
                    if (pixel.x < 0.0 || pixel.x >= (double)w || pixel.y < 0.0 || pixel.y >= (double)h) continue;
                    size_t px = (size_t)pixel.x, py = (size_t)pixel.y;
                    size_t sx = std::min(side - 1, (size_t)((pixel.x - (double)px) * (double)side));
                    size_t sy = std::min(side - 1, (size_t)((pixel.y - (double)py) * (double)side));
                    depth_test((py * w + px) * spp + sy * side + sx, pr.depth, pr.color, depth.data(), color.data(), st);
                } else {
                    write_block(pixel, fp, w, h, (int64_t)side, pr.depth, pr.color, depth.data(), color.data(), st);
                }
            }
        }
        resolve_set(w, h, spp, depth.data(), color.data(), bg, accum);
    }
}

void render_monte_carlo(const Gaussian3D* scene, size_t n, Camera cam, size_t w, size_t h, size_t side, size_t sets, V3 bg,
                        uint32_t base_seed, const MCOptions& opt, V3* img, RenderStats& st, int threads) {
    cam = with_default_pp(cam, w, h);
    side = std::min(std::max(side, (size_t)1), (size_t)4);
    std::vector<Projected> proj;
    for (size_t i = 0; i < n; ++i) {
        Projected p;
        if (project(scene[i], cam, p)) proj.push_back(p);
    }
    std::vector<uint32_t> footprint(proj.size(), 1);
    std::vector<M2> sample_cov(proj.size());
    for (size_t g = 0; g < proj.size(); ++g) {
        const Projected& pr = proj[g];
        sample_cov[g] = pr.cov2d;
        uint32_t fp = std::max(opt.footprint_subpixels, 1u);
        if (opt.adaptive_kappa > 0.0) {
            double tr = pr.cov2d.x.x + pr.cov2d.y.y;
            double disc = sqrt(std::max(0.25 * tr * tr - pr.det, 0.0));
            double smin = sqrt(std::max(0.5 * tr - disc, 0.0));
            fp = adaptive_footprint(smin * (double)side, opt.adaptive_kappa, opt.footprint_max);
        }
        footprint[g] = fp;
        if (opt.compensate_blur && fp > 1) {
            double v = ((double)fp / (double)side) * ((double)fp / (double)side) / 12.0;
            M2 sh = pr.cov2d;
            sh.x.x -= v;
            sh.y.y -= v;
            double t = sh.x.x + sh.y.y, d = det2(sh);
            if (d > 0.0 && t > 0.0 && 0.5 * t - sqrt(std::max(0.25 * t * t - d, 0.0)) >= v) sample_cov[g] = sh;
        }
    }
    for (size_t i = 0; i < w * h; ++i) img[i] = {0, 0, 0};
    st = {0, 0, 0};
    threads = std::max(1, std::min(threads, (int)sets));
    if (threads == 1) {
        mc_sets(proj, footprint, sample_cov, w, h, side, bg, base_seed, opt, 0, sets, img, st);
    } else {
        std::vector<std::vector<V3>> part(threads, std::vector<V3>(w * h, V3{0, 0, 0}));
        std::vector<RenderStats> pst(threads, RenderStats{0, 0, 0});
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t) {
            size_t lo = sets * t / threads, hi = sets * (t + 1) / threads;
            th.emplace_back([&, t, lo, hi] { mc_sets(proj, footprint, sample_cov, w, h, side, bg, base_seed, opt, lo, hi, part[t].data(), pst[t]); });
        }
        for (auto& x : th) x.join();
        for (int t = 0; t < threads; ++t) {
            for (size_t i = 0; i < w * h; ++i) img[i] = add(img[i], part[t][i]);
            st.points += pst[t].points;
            st.candidates += pst[t].candidates;
            st.subpixel_writes += pst[t].subpixel_writes;
        }
    }
    for (size_t i = 0; i < w * h; ++i) img[i] = mul(img[i], 1.0 / (double)sets);
}

struct POptions {  // oracle.rs:317-350
    int level, rule, radial_correction;
    double base_k, reference_pixel_length, near_z;
    int low_pass_jitter, centre_depth, linearized_projection;
    double density_scale;
    int per_particle_seed;
    // Per-splat cap on the candidate count as the GPU applies it (gps_splat.wgsl:597-602);
    // 0xFFFFFFFF = none (the oracle's own behaviour).
    uint32_t max_points_per_splat;
};
static M3 cholesky_3d(const M3& c) {  // oracle.rs:352-361
    double a00 = c.c[0].x, a10 = c.c[0].y, a20 = c.c[0].z, a11 = c.c[1].y, a21 = c.c[1].z, a22 = c.c[2].z;
    double l00 = sqrt(std::max(a00, 1e-30));
    double l10 = a10 / l00, l20 = a20 / l00;
    double l11 = sqrt(std::max(a11 - l10 * l10, 1e-30));
    double l21 = (a21 - l20 * l10) / l11;
    double l22 = sqrt(std::max(a22 - l20 * l20 - l21 * l21, 1e-30));
    return {{{l00, l10, l20}, {0.0, l11, l21}, {0.0, 0.0, l22}}};
}
struct Prep { uint32_t index; V3 pos; Projected pr; M3 l3; M2 cov2d_inv; M3 jw; double lambda; };

static void particle_sets(const std::vector<Prep>& preps, const Camera& cam, const Pinhole& pin, V3 forward, double jitter,
                          size_t w, size_t h, size_t side, V3 bg, uint32_t base_seed, const POptions& opt, size_t set_lo,
                          size_t set_hi, V3* accum, RenderStats& st) {
    size_t spp = side * side, n_sub = w * h * spp;
    std::vector<double> depth(n_sub);
    std::vector<V3> color(n_sub);
    for (size_t s = set_lo; s < set_hi; ++s) {
        std::fill(depth.begin(), depth.end(), 1e300);
        std::fill(color.begin(), color.end(), V3{0, 0, 0});
        for (size_t gid = 0; gid < preps.size(); ++gid) {
            const Prep& p = preps[gid];
            if (p.lambda <= 0.0) continue;
            uint32_t set_seed = base_seed + (uint32_t)s;
            RandStream rng = opt.per_particle_seed ? RandStream(particle_seed(true, p.index, 0, set_seed))
                                                   : RandStream(particle_seed(true, (uint32_t)gid, 1, set_seed));
            int32_t n = poisson_sample(p.lambda, rng);
            st.candidates += (double)n;
            if ((uint32_t)n > opt.max_points_per_splat) n = (int32_t)opt.max_points_per_splat;
            for (int32_t k = 0; k < n; ++k) {
                if (opt.per_particle_seed) rng = RandStream(particle_seed(true, p.index, (uint32_t)k + 1u, set_seed));
                // MSVC right-to-left argument order: z, y, x (oracle.rs:445-451)
                double uz = rng.normal(), uy = rng.normal(), ux = rng.normal();
                V3 world = add(p.pos, mv(p.l3, V3{ux, uy, uz}));
                V2 pixel;
                double d;
                if (opt.linearized_projection) {
                    V3 off = mv(p.jw, sub(world, p.pos));
                    pixel = {p.pr.mean.x + off.x, p.pr.mean.y + off.y};
                    d = p.pr.depth + dot(forward, sub(world, p.pos));
                } else {
                    V3 cp = world_to_camera(pin, world);
                    if (cp.z <= opt.near_z) continue;
                    pixel = {cam.fx * cp.x / cp.z + cam.cx, cam.fy * cp.y / cp.z + cam.cy};
                    d = cp.z;
                }
                if (jitter > 0.0) {
                    double jy = rng.normal(), jx = rng.normal();
                    pixel = {pixel.x + jitter * jx, pixel.y + jitter * jy};
                }
                if (opt.radial_correction) {
                    V2 dv = {pixel.x - p.pr.mean.x, pixel.y - p.pr.mean.y};
                    V2 t = mv2(p.cov2d_inv, dv);
                    double r2 = dv.x * t.x + dv.y * t.y;
                    if (rng.next() >= radial_keep_probability(p.pr.opacity, r2)) continue;
                }
                if (opt.centre_depth) d = p.pr.depth;
                st.points += 1.0;
                if (pixel.x < 0.0 || pixel.x >= (double)w || pixel.y < 0.0 || pixel.y >= (double)h) continue;
                size_t px = (size_t)pixel.x, py = (size_t)pixel.y;
                size_t sx = std::min(side - 1, (size_t)((pixel.x - (double)px) * (double)side));
                size_t sy = std::min(side - 1, (size_t)((pixel.y - (double)py) * (double)side));
                depth_test((py * w + px) * spp + sy * side + sx, d, p.pr.color, depth.data(), color.data(), st);
            }
        }
        resolve_set(w, h, spp, depth.data(), color.data(), bg, accum);
    }
}

// render_particles_3d (oracle.rs:374-499)
void render_particles_3d(const Gaussian3D* scene, size_t n, Camera cam, size_t w, size_t h, size_t side, size_t sets, V3 bg,
                         uint32_t base_seed, const POptions& opt, V3* img, RenderStats& st, int threads) {
    cam = with_default_pp(cam, w, h);
    side = std::min(std::max(side, (size_t)1), (size_t)4);
    size_t spp = side * side;
    Pinhole pin = to_pinhole(cam);
    V3 centre = {0, 0, 0};
    for (size_t i = 0; i < n; ++i) centre = add(centre, scene[i].pos);
    if (n) centre = mul(centre, 1.0 / (double)n);
    double object_depth = world_to_camera(pin, centre).z;
    std::vector<Prep> preps;
    for (size_t si = 0; si < n; ++si) {
        const Gaussian3D& g = scene[si];
        Projected pr;
        if (!project(g, cam, pr)) continue;
        M3 cov3 = covariance_3d(g.log_scale, g.rot);
        M3 l3 = cholesky_3d(cov3);
        V3 cm = world_to_camera(pin, g.pos);
        double iz = 1.0 / cm.z;
        V3 jx = {cam.fx * iz, 0.0, -cam.fx * cm.x * iz * iz};
        V3 jy = {0.0, cam.fy * iz, -cam.fy * cm.y * iz * iz};
        M3 wt = transpose(cam.view_rot);
        V3 rx = mv(wt, jx), ry = mv(wt, jy);
        M3 jw = {{{rx.x, ry.x, 0.0}, {rx.y, ry.y, 0.0}, {rx.z, ry.z, 0.0}}};
        CalIn in = {object_depth, cm.z, cam.fx, cam.fy, opt.near_z, opt.reference_pixel_length, projected_footprint_area(pr.cov2d), (double)spp};
        double lambda = calibrated_count(opt.level, opt.rule, pr.opacity, opt.base_k, opt.density_scale, in);
        preps.push_back({(uint32_t)si, g.pos, pr, l3, inverse2(pr.cov2d), jw, lambda});
    }
    V3 forward = transpose(cam.view_rot).c[2];
    double jitter = opt.low_pass_jitter ? sqrt(std::max(cam.low_pass, 0.0)) : 0.0;
    for (size_t i = 0; i < w * h; ++i) img[i] = {0, 0, 0};
    st = {0, 0, 0};
    threads = std::max(1, std::min(threads, (int)sets));
    if (threads == 1) {
        particle_sets(preps, cam, pin, forward, jitter, w, h, side, bg, base_seed, opt, 0, sets, img, st);
    } else {
        std::vector<std::vector<V3>> part(threads, std::vector<V3>(w * h, V3{0, 0, 0}));
        std::vector<RenderStats> pst(threads, RenderStats{0, 0, 0});
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t) {
            size_t lo = sets * t / threads, hi = sets * (t + 1) / threads;
            th.emplace_back([&, t, lo, hi] { particle_sets(preps, cam, pin, forward, jitter, w, h, side, bg, base_seed, opt, lo, hi, part[t].data(), pst[t]); });
        }
        for (auto& x : th) x.join();
        for (int t = 0; t < threads; ++t) {
            for (size_t i = 0; i < w * h; ++i) img[i] = add(img[i], part[t][i]);
            st.points += pst[t].points;
            st.candidates += pst[t].candidates;
            st.subpixel_writes += pst[t].subpixel_writes;
        }
    }
    for (size_t i = 0; i < w * h; ++i) img[i] = mul(img[i], 1.0 / (double)std::max(sets, (size_t)1));
}

double psnr(const V3* a, const V3* b, size_t n) {  // oracle.rs:503-514
    if (n == 0) return 0.0;
    double mse = 0.0;
    for (size_t i = 0; i < n; ++i) {
        V3 d = sub(a[i], b[i]);
        mse += dot(d, d);
    }
    mse /= (double)(n * 3);
    return mse <= 1e-20 ? 120.0 : 10.0 * log10(1.0 / mse);
}
double ssim(const V3* a, const V3* b, size_t w, size_t h) {  // oracle.rs:517-559
    auto lum = [](V3 c) { return 0.299 * c.x + 0.587 * c.y + 0.114 * c.z; };
    const double c1 = 0.01 * 0.01, c2 = 0.03 * 0.03;
    double total = 0.0;
    size_t count = 0;
    for (size_t y0 = 0; y0 + 8 <= h; y0 += 4)
        for (size_t x0 = 0; x0 + 8 <= w; x0 += 4) {
            double ma = 0, mb = 0;
            for (size_t y = 0; y < 8; ++y)
                for (size_t x = 0; x < 8; ++x) {
                    size_t i = (y0 + y) * w + x0 + x;
                    ma += lum(a[i]);
                    mb += lum(b[i]);
                }
            ma /= 64.0;
            mb /= 64.0;
            double va = 0, vb = 0, cov = 0;
            for (size_t y = 0; y < 8; ++y)
                for (size_t x = 0; x < 8; ++x) {
                    size_t i = (y0 + y) * w + x0 + x;
                    double da = lum(a[i]) - ma, db = lum(b[i]) - mb;
                    va += da * da;
                    vb += db * db;
                    cov += da * db;
                }
            va /= 63.0;
            vb /= 63.0;
            cov /= 63.0;
            total += ((2.0 * ma * mb + c1) * (2.0 * cov + c2)) / ((ma * ma + mb * mb + c1) * (va + vb + c2));
            count += 1;
        }
    return count ? total / (double)count : 1.0;
}

// ------------------------------------------------------------------ camera.rs / OracleCamera::look_at
Camera look_at(V3 eye, V3 target, V3 up, double fov_y, uint32_t w, uint32_t h) {  // oracle.rs:53-70
    V3 f = normalize(sub(target, eye));
    V3 right = normalize(cross(f, up));
    V3 down = cross(f, right);
    M3 cols = {{right, down, f}};
    Camera c;
    c.view_rot = transpose(cols);
    c.view_pos = eye;
    double focal = 0.5 * (double)h / tan(0.5 * fov_y);
    c.fx = c.fy = focal;
    c.cx = 0.5 * (double)w;
    c.cy = 0.5 * (double)h;
    c.low_pass = 0.3;
    return c;
}
V3 orbit_eye(V3 target, double distance, double yaw, double pitch, V3 up) {  // camera.rs:31-40
    up = normalize(up);
    V3 helper = fabs(up.x) < 0.9 ? V3{1, 0, 0} : V3{0, 0, 1};
    V3 a = normalize(cross(up, helper));
    V3 b = cross(up, a);
    V3 horiz = add(mul(a, cos(yaw)), mul(b, sin(yaw)));
    V3 dir = add(mul(horiz, cos(pitch)), mul(up, sin(pitch)));
    return add(target, mul(dir, distance));
}

}  // namespace o1

// ============================================================================ C entry points
using namespace o1;

// Flat scene record for ctypes: pos[3], log_scale[3], rot xyzw[4], opacity, color[3] = 14 doubles.
static std::vector<Gaussian3D> unpack(const double* s, size_t n) {
    std::vector<Gaussian3D> v(n);
    for (size_t i = 0; i < n; ++i) {
        const double* r = s + i * 14;
        v[i] = {{r[0], r[1], r[2]}, {r[3], r[4], r[5]}, {r[6], r[7], r[8], r[9]}, r[10], {r[11], r[12], r[13]}};
    }
    return v;
}
// Flat camera: view_rot row-major[9], view_pos[3], fx, fy, cx, cy, low_pass = 17 doubles.
static Camera unpack_cam(const double* c) {
    Camera k;
    k.view_rot = from_rows(c);
    k.view_pos = {c[9], c[10], c[11]};
    k.fx = c[12]; k.fy = c[13]; k.cx = c[14]; k.cy = c[15]; k.low_pass = c[16];
    return k;
}

extern "C" {

double o1_dilog(double x) { return dilog(x); }
double o1_inv_dilog(double x) { return inv_dilog(x); }
double o1_sigmoid(double x) { return sigmoid(x); }
double o1_expected_point_count(double det, double o) { return expected_point_count(det, o); }
uint32_t o1_pcg_hash(uint32_t v) { return pcg_hash(v); }
uint32_t o1_particle_seed(int fv, uint32_t s, uint32_t k, uint32_t f) { return particle_seed(fv != 0, s, k, f); }
uint32_t o1_ordered_depth_key(float d) { return ordered_depth_key(d); }
float o1_ordered_depth_key_inverse(uint32_t k) { return ordered_depth_key_inverse(k); }
double o1_sample_corrected_radius(double o, double u) { return sample_corrected_radius(o, u); }
double o1_radial_keep_probability(double o, double r2) { return radial_keep_probability(o, r2); }
double o1_calibrated_count(int level, int rule, double o, double base_k, double density, const double* in8) {
    CalIn in = {in8[0], in8[1], in8[2], in8[3], in8[4], in8[5], in8[6], in8[7]};
    return calibrated_count(level, rule, o, base_k, density, in);
}
void o1_radius_lut(float* out) { radius_lut(out); }
double o1_radius_from_lut(const float* lut, double o, double u) { return radius_from_lut(lut, o, u); }
// Poisson draws: out[i] for i < n from one RandStream(seed).
void o1_poisson_stream(double lambda, uint32_t seed, int32_t* out, size_t n) {
    RandStream r(seed);
    for (size_t i = 0; i < n; ++i) out[i] = poisson_sample(lambda, r);
}
// covariance_2d of (log_scale, rot xyzw) at mean for a pinhole (fx, fy, tan 1) with identity pose: out[4] col-major
void o1_covariance_2d(const double* log_scale, const double* rot_xyzw, const double* mean, double fx, double fy,
                      double tan_fov, double low_pass, double* out) {
    Pinhole pin = {{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}}, {0, 0, 0}, fx, fy, tan_fov, tan_fov};
    M3 c3 = covariance_3d({log_scale[0], log_scale[1], log_scale[2]}, {rot_xyzw[0], rot_xyzw[1], rot_xyzw[2], rot_xyzw[3]});
    M2 c2 = covariance_2d(c3, {mean[0], mean[1], mean[2]}, pin, low_pass);
    out[0] = c2.x.x; out[1] = c2.x.y; out[2] = c2.y.x; out[3] = c2.y.y;
}
void o1_eval_sh(int degree, const double* dc, const double* rest, const double* dir, int stride, double* out) {
    V3 r = eval_sh(degree, {dc[0], dc[1], dc[2]}, rest, {dir[0], dir[1], dir[2]}, stride);
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void o1_render_analytic(const double* scene, size_t n, const double* cam, size_t w, size_t h, const double* bg, double* img) {
    auto s = unpack(scene, n);
    render_analytic(s.data(), n, unpack_cam(cam), w, h, {bg[0], bg[1], bg[2]}, (V3*)img);
}
// opt: footprint_subpixels, adaptive_kappa, footprint_max, compensate_blur, density_scale, per_particle_seed, max_points
void o1_render_monte_carlo(const double* scene, size_t n, const double* cam, size_t w, size_t h, size_t side, size_t sets,
                           const double* bg, uint32_t seed, const double* opt7, double* img, double* stats3, int threads) {
    auto s = unpack(scene, n);
    MCOptions o = {(uint32_t)opt7[0], opt7[1], (uint32_t)opt7[2], (int)opt7[3], opt7[4], (int)opt7[5],
                   opt7[6] >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)opt7[6]};
    RenderStats st;
    render_monte_carlo(s.data(), n, unpack_cam(cam), w, h, side, sets, {bg[0], bg[1], bg[2]}, seed, o, (V3*)img, st, threads);
    stats3[0] = st.points; stats3[1] = st.candidates; stats3[2] = st.subpixel_writes;
}
// opt: level, rule, radial, base_k, refl, near, jitter, centre, linearized, density, per_particle_seed, cap
void o1_render_particles_3d(const double* scene, size_t n, const double* cam, size_t w, size_t h, size_t side, size_t sets,
                            const double* bg, uint32_t seed, const double* opt12, double* img, double* stats3, int threads) {
    auto s = unpack(scene, n);
    POptions o = {(int)opt12[0], (int)opt12[1], (int)opt12[2], opt12[3], opt12[4], opt12[5],
                  (int)opt12[6], (int)opt12[7], (int)opt12[8], opt12[9], (int)opt12[10],
                  opt12[11] >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)opt12[11]};
    RenderStats st;
    render_particles_3d(s.data(), n, unpack_cam(cam), w, h, side, sets, {bg[0], bg[1], bg[2]}, seed, o, (V3*)img, st, threads);
    stats3[0] = st.points; stats3[1] = st.candidates; stats3[2] = st.subpixel_writes;
}
double o1_psnr(const double* a, const double* b, size_t n) { return psnr((const V3*)a, (const V3*)b, n); }
double o1_ssim(const double* a, const double* b, size_t w, size_t h) { return ssim((const V3*)a, (const V3*)b, w, h); }
void o1_look_at(const double* eye, const double* target, const double* up, double fov_y, uint32_t w, uint32_t h, double* cam17) {
    Camera c = look_at({eye[0], eye[1], eye[2]}, {target[0], target[1], target[2]}, {up[0], up[1], up[2]}, fov_y, w, h);
    M3 r = transpose(c.view_rot);  // columns of the transpose = rows of view_rot
    for (int i = 0; i < 3; ++i) {
        cam17[i * 3 + 0] = r.c[i].x;
        cam17[i * 3 + 1] = r.c[i].y;
        cam17[i * 3 + 2] = r.c[i].z;
    }
    cam17[9] = c.view_pos.x; cam17[10] = c.view_pos.y; cam17[11] = c.view_pos.z;
    cam17[12] = c.fx; cam17[13] = c.fy; cam17[14] = c.cx; cam17[15] = c.cy; cam17[16] = c.low_pass;
}
void o1_orbit_eye(const double* target, double distance, double yaw, double pitch, const double* up, double* eye) {
    V3 e = orbit_eye({target[0], target[1], target[2]}, distance, yaw, pitch, {up[0], up[1], up[2]});
    eye[0] = e.x; eye[1] = e.y; eye[2] = e.z;
}

}  // extern "C"
