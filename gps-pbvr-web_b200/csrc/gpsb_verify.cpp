// gpsb-verify: command-line runner over the C ABI, restating the reference's native CLI
// (crates/gps-verify/src/main.rs:105-178).
//   gpsb-verify bench-ply <file.ply> [WxH] [spp_side]   per-ensemble GPU time of GPS, PBVR Ext C3+R
//                                                       and ScreenOccupancy at near/mid/far framings
//                                                       (main.rs:106-148; MAXPTS = per-splat cap)
//   gpsb-verify bench                                   splat-parallel vs particle-parallel timing on
//                                                       the synthetic shell scene (main.rs:22-103)
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gpsb200.h"

static void die(gpsb_renderer* r, gpsb_status s, const char* what) {
    if (s != GPSB_OK) {
        fprintf(stderr, "%s failed: %s\n", what, r ? gpsb_last_error(r) : gpsb_last_error(nullptr));
        exit(1);
    }
}

static uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}

// main.rs:22-53: n Gaussians on three sphere shells plus `big` very large splats
static std::vector<gpsb_gaussian> shell_scene(size_t n, size_t big) {
    uint32_t s = 12345;
    auto rnd = [&]() { s = pcg(s); return (float)s * (1.0f / 4294967296.0f); };
    std::vector<gpsb_gaussian> v;
    for (size_t i = 0; i < n; ++i) {
        float u = rnd() * 6.2831853f, w = rnd() * 2.0f - 1.0f;
        float ring = 0.6f + 0.25f * (float)(i % 3);
        float x = ring * std::sqrt(1.0f - w * w) * std::cos(u), y = w * ring, z = ring * std::sqrt(1.0f - w * w) * std::sin(u);
        float sc = std::log(0.05f + 0.05f * rnd());
        gpsb_gaussian g = {{x, y, z, 0.5f + 0.45f * rnd()}, {sc, sc, sc, 0}, {1, 0, 0, 0},
                           {0.5f + 0.4f * x, 0.5f + 0.4f * y, 0.5f + 0.4f * z, 0}};
        v.push_back(g);
    }
    for (size_t i = 0; i < big; ++i) {
        float sc = std::log(0.9f + 0.2f * (float)i);
        gpsb_gaussian g = {{0, 0, 0, 0.8f}, {sc, sc, std::log(0.1f), 0}, {1, 0, 0, 0}, {0.3f, 0.3f, 0.35f, 0}};
        v.push_back(g);
    }
    return v;
}

static double time_ms(gpsb_renderer* r, const gpsb_camera& cam, const gpsb_params& p, int reps) {
    die(r, gpsb_render_ensembles(r, &cam, &p, 1, 1), "warm-up render");
    die(r, gpsb_sync(r), "sync");
    die(r, gpsb_reset_stats(r), "reset stats");
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < reps; ++i) {
        die(r, gpsb_render_ensembles(r, &cam, &p, 100 + i, 1), "render");
        die(r, gpsb_sync(r), "sync");
    }
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / reps;
}

static int bench() {
    struct Case { const char* label; size_t n, big; uint32_t w, h, spp; bool primitive; };
    Case cases[] = {{"320x180 spp1, 600 splats", 600, 0, 320, 180, 1, true},
                    {"640x360 spp1, 600 splats", 600, 0, 640, 360, 1, true},
                    {"640x360 spp4, 600 splats", 600, 0, 640, 360, 2, true},
                    {"640x360 spp1, 600 + 2 huge splats", 600, 2, 640, 360, 1, false},
                    {"640x360 spp1, 20000 splats", 20000, 0, 640, 360, 1, true}};
    printf("%-40s %11s %12s %13s\n", "case (ms per ensemble, lower is better)", "points/ens", "splat-par", "particle-par");
    for (const Case& c : cases) {
        gpsb_renderer* r = nullptr;
        die(nullptr, gpsb_create(0, c.w, c.h, c.spp, &r), "create");
        auto sc = shell_scene(c.n, c.big);
        die(r, gpsb_set_gaussians(r, sc.data(), sc.size()), "set_gaussians");
        double target[3] = {0, 0, 0}, up[3] = {0, 1, 0};
        double dist = (1.0 / std::sin(0.45)) * 1.25;
        gpsb_camera cam;
        die(r, gpsb_orbit_camera(target, dist, 0.6, 0.25, up, 0.9, c.w, c.h, &cam), "camera");
        double ms[2] = {NAN, NAN};
        uint64_t points = 0;
        for (int k = 0; k < 2; ++k) {
            if (k == 0 && !c.primitive) continue;
            gpsb_params p;
            gpsb_params_default(&p);
            p.spp_side = c.spp;
            p.path = k == 0 ? GPSB_PATH_PRIMITIVE : GPSB_PATH_PARTICLE;
            ms[k] = time_ms(r, cam, p, 12);
            gpsb_stats st;
            die(r, gpsb_read_stats(r, &st), "stats");
            points = st.points / 12;
        }
        if (c.primitive)
            printf("%-40s %11llu %10.3fms %11.3fms  (%.1fx)\n", c.label, (unsigned long long)points, ms[0], ms[1], ms[0] / ms[1]);
        else
            printf("%-40s %11llu %12s %11.3fms\n", c.label, (unsigned long long)points, "(skipped)", ms[1]);
        gpsb_destroy(r);
    }
    return 0;
}

static int bench_ply(const char* path, const char* size, uint32_t spp) {
    FILE* f = fopen(path, "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); return 1; }
    std::vector<uint8_t> bytes;
    uint8_t buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, f)) > 0) bytes.insert(bytes.end(), buf, buf + got);
    fclose(f);
    size_t n = 0;
    uint32_t deg = 0;
    if (gpsb_load_ply(bytes.data(), bytes.size(), &n, &deg, nullptr, nullptr) != GPSB_OK) {
        fprintf(stderr, "load ply: %s\n", gpsb_ply_last_error());
        return 1;
    }
    size_t per = deg ? (deg + 1) * (deg + 1) - 1 : 0;
    std::vector<gpsb_gaussian> g(n);
    std::vector<float> sh(n * 3 * per);
    if (gpsb_load_ply(bytes.data(), bytes.size(), &n, &deg, g.data(), sh.empty() ? nullptr : sh.data()) != GPSB_OK) {
        fprintf(stderr, "load ply: %s\n", gpsb_ply_last_error());
        return 1;
    }
    uint32_t w = 480, h = 270;
    if (sscanf(size, "%ux%u", &w, &h) != 2) { w = 480; h = 270; }
    gpsb_renderer* r = nullptr;
    die(nullptr, gpsb_create(0, w, h, spp, &r), "create");
    printf("%s | %zu Gaussians, SH degree %u\n", gpsb_version(), n, deg);
    if (deg) die(r, gpsb_set_gaussians_sh(r, g.data(), n, sh.data(), sh.size(), deg), "scene");
    else die(r, gpsb_set_gaussians(r, g.data(), n), "scene");
    double centre[3], rad = 1.0;
    die(r, gpsb_robust_sphere(g.data(), n, centre, &rad), "robust sphere");
    const char* env = getenv("MAXPTS");
    uint32_t maxpts = env ? (uint32_t)strtoul(env, nullptr, 10) : 16384u;
    printf("%-34s %13s %10s %12s\n", "view / method", "points/ens", "ms/ens", "truncated");
    struct View { const char* name; double mul; } views[] = {{"near (x1.25)", 1.0}, {"mid (x2.3)", 1.85}, {"far (x4)", 3.2}};
    struct Meth { const char* name; uint32_t method, cal, radial; } meths[] = {
        {"GPS", GPSB_METHOD_GPS, GPSB_CAL_PER_SPLAT_FOOTPRINT, 0},
        {"PBVR Ext C3+R", GPSB_METHOD_EXTINCTION, GPSB_CAL_PER_SPLAT_FOOTPRINT, 1},
        {"Screen occupancy", GPSB_METHOD_SCREEN_OCCUPANCY, GPSB_CAL_NONE, 0}};
    double up[3] = {0, -1, 0};
    for (const View& v : views) {
        double dist = (std::max(rad, 1e-6) / std::sin(0.45)) * 1.25 * v.mul;
        gpsb_camera cam;
        die(r, gpsb_orbit_camera(centre, dist, 0.6, 0.25, up, 0.9, w, h, &cam), "camera");
        for (const Meth& m : meths) {
            gpsb_params p;
            gpsb_params_default(&p);
            p.spp_side = spp;
            p.max_points_per_splat = maxpts;
            p.method = m.method;
            p.pbvr.calibration = m.cal;
            p.pbvr.radial_correction = m.radial;
            double ms = time_ms(r, cam, p, 6);
            gpsb_stats st;
            die(r, gpsb_read_stats(r, &st), "stats");
            char label[96];
            snprintf(label, sizeof label, "%s %s", v.name, m.name);
            printf("%-34s %13llu %8.2fms %12llu\n", label, (unsigned long long)(st.points / 6), ms,
                   (unsigned long long)(st.truncated_splats / 6));
            if (m.method == GPSB_METHOD_SCREEN_OCCUPANCY)
                printf("    candidate tests/ens=%llu skipped=%llu orphan=%llu\n", (unsigned long long)(st.candidates / 6),
                       (unsigned long long)st.skipped_ensembles, (unsigned long long)st.orphan_subpixels);
        }
    }
    gpsb_destroy(r);
    return 0;
}

int main(int argc, char** argv) {
    std::string which = argc > 1 ? argv[1] : "";
    if (which == "bench-ply") {
        if (argc < 3) { fprintf(stderr, "usage: gpsb-verify bench-ply <file.ply> [WxH] [spp_side]\n"); return 2; }
        return bench_ply(argv[2], argc > 3 ? argv[3] : "480x270", argc > 4 ? (uint32_t)atoi(argv[4]) : 1u);
    }
    if (which == "bench") return bench();
    fprintf(stderr, "usage: gpsb-verify bench-ply <file.ply> [WxH] [spp_side] | gpsb-verify bench\n"
                    "(the correctness phases of the reference CLI are the pytest suite: pytest tests -m gpu)\n");
    return 2;
}
