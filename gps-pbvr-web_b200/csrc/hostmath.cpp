// Host-side set-up maths of the renderer: the corrected-radius table the particle kernels read
// (gps_core::radius_lut, crates/gps-core/src/lib.rs:611-636, built on the host at renderer
// creation exactly like gps-render does), and the camera helpers of crates/gps-core/src/camera.rs
// and OracleCamera::look_at (oracle.rs:53-70) that callers use to build gpsb_camera values.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/gpsb200.h"

namespace gpsb {

static const double kDilogOne = 1.6449340668482264;  // pi^2 / 6

static double li2_series(double x) {
    double term = x, sum = x;
    for (int k = 2; k < 1000; ++k) {
        term *= x;
        double add = term / ((double)k * (double)k);
        sum += add;
        if (fabs(add) < 1e-18 * fabs(sum)) break;
    }
    return sum;
}
// Li2 on [0, 1] (the table only needs non-negative arguments; lib.rs:193-212)
static double li2(double x) {
    if (x >= 1.0) return kDilogOne;
    if (x <= 0.0) return 0.0;
    if (x <= 0.5) return li2_series(x);
    return kDilogOne - log(x) * log(1.0 - x) - li2_series(1.0 - x);
}
// Safeguarded Newton inverse of Li2 on [0, 1) (lib.rs:219-248)
static double li2_inverse(double target) {
    double top;
    uint64_t b;
    memcpy(&b, &kDilogOne, 8);
    b -= 1;
    memcpy(&top, &b, 8);
    target = std::min(std::max(target, 0.0), top);
    if (target <= 0.0) return 0.0;
    double lo = 0.0, hi = 1.0, y = target / kDilogOne;
    for (int it = 0; it < 40; ++it) {
        double f = li2(y) - target;
        if (f > 0.0) hi = y; else lo = y;
        double d = (y > 1e-12 && y < 1.0 - 1e-15) ? -log(1.0 - y) / y : 1.0;
        double ny = y - f / d;
        if (!(ny > lo && ny < hi)) ny = 0.5 * (lo + hi);
        if (fabs(ny - y) <= 1e-14 * (1.0 + y)) return ny;
        y = ny;
    }
    return y;
}
// Whitened radius of F(r) = 1 - Li2(o e^{-r^2/2}) / Li2(o) at quantile u (lib.rs:522-536)
static double corrected_radius(double opacity, double u) {
    double o = std::min(std::max(opacity, 0.0), 1.0);
    if (o <= 0.0) return 0.0;
    u = std::min(std::max(u, 0.0), 1.0);
    double y = std::min(li2_inverse((1.0 - u) * li2(o)), o);
    if (y <= 0.0) return 40.0;
    return sqrt(std::max(-2.0 * log(y / o), 0.0));
}

// 65 opacity rows (o = 1 - (1 - x)^2) x 129 nodes in w = sqrt(-ln(1 - u)) on [0, sqrt 17].
void host_radius_lut(float* t) {
    for (int i = 0; i < 65; ++i) {
        double x = (double)i / 64.0;
        double o = std::min(std::max(1.0 - (1.0 - x) * (1.0 - x), 1e-6), 1.0);
        for (int j = 0; j < 129; ++j) {
            double w = (double)j * sqrt(17.0) / 128.0;
            double u = -expm1(-w * w);
            t[i * 129 + j] = (float)corrected_radius(o, u);
        }
    }
}

struct D3 { double x, y, z; };
static D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static D3 mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static D3 cross(D3 a, D3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
static D3 normalize(D3 a) { return mul(a, 1.0 / sqrt(a.x * a.x + a.y * a.y + a.z * a.z)); }

}  // namespace gpsb

using namespace gpsb;

extern "C" {

gpsb_status gpsb_radius_lut(float* out) {
    if (!out) return GPSB_ERR_INVALID_ARGUMENT;
    host_radius_lut(out);
    return GPSB_OK;
}

gpsb_status gpsb_camera_look_at(const double eye[3], const double target[3], const double up[3], double fov_y, uint32_t w,
                                uint32_t h, gpsb_camera* out) {
    if (!eye || !target || !up || !out || w == 0 || h == 0) return GPSB_ERR_INVALID_ARGUMENT;
    D3 e = {eye[0], eye[1], eye[2]}, t = {target[0], target[1], target[2]}, u = {up[0], up[1], up[2]};
    D3 f = normalize(sub(t, e));
    D3 right = normalize(cross(f, u));
    D3 down = cross(f, right);
    // rows of view_rot are the camera axes in world space
    double R[9] = {right.x, right.y, right.z, down.x, down.y, down.z, f.x, f.y, f.z};
    memcpy(out->view_rot, R, sizeof R);
    out->view_pos[0] = e.x;
    out->view_pos[1] = e.y;
    out->view_pos[2] = e.z;
    double focal = 0.5 * (double)h / tan(0.5 * fov_y);
    out->focal_x = out->focal_y = focal;
    out->cx = 0.5 * (double)w;
    out->cy = 0.5 * (double)h;
    out->low_pass = 0.3;
    return GPSB_OK;
}

gpsb_status gpsb_orbit_camera(const double target[3], double distance, double yaw, double pitch, const double up[3],
                              double fov_y, uint32_t w, uint32_t h, gpsb_camera* out) {
    if (!target || !up || !out) return GPSB_ERR_INVALID_ARGUMENT;
    D3 u = normalize(D3{up[0], up[1], up[2]});
    D3 helper = fabs(u.x) < 0.9 ? D3{1, 0, 0} : D3{0, 0, 1};
    D3 a = normalize(cross(u, helper));
    D3 b = cross(u, a);
    D3 horiz = add(mul(a, cos(yaw)), mul(b, sin(yaw)));
    D3 dir = add(mul(horiz, cos(pitch)), mul(u, sin(pitch)));
    D3 t = {target[0], target[1], target[2]};
    D3 eye = add(t, mul(dir, distance));
    double e3[3] = {eye.x, eye.y, eye.z};
    return gpsb_camera_look_at(e3, target, up, fov_y, w, h, out);
}

gpsb_status gpsb_robust_sphere(const gpsb_gaussian* s, size_t n, double centre[3], double* radius) {
    if (!s || n == 0 || !centre || !radius) return GPSB_ERR_INVALID_ARGUMENT;
    std::vector<double> v(n);
    for (int ax = 0; ax < 3; ++ax) {
        for (size_t i = 0; i < n; ++i) v[i] = (double)s[i].pos_opacity[ax];
        std::nth_element(v.begin(), v.begin() + n / 2, v.end());
        centre[ax] = v[n / 2];
    }
    for (size_t i = 0; i < n; ++i) {
        double dx = s[i].pos_opacity[0] - centre[0], dy = s[i].pos_opacity[1] - centre[1], dz = s[i].pos_opacity[2] - centre[2];
        v[i] = sqrt(dx * dx + dy * dy + dz * dz);
    }
    size_t k = std::min((size_t)((double)n * 0.75), n - 1);
    std::nth_element(v.begin(), v.begin() + k, v.end());
    *radius = v[k];
    return GPSB_OK;
}

}  // extern "C"
