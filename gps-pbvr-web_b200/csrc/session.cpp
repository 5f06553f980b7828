// Frame-loop policy of the reference's viewer (crates/gps-web/src/lib.rs:437-697, Viewer::frame and
// its setters), headless: which hot-path variant runs each tick (GPS particles, the depth-sorted
// path, or a demand probe first), how many ensembles (manual or adaptive LOD), the point-budget
// density factor, the moving-camera particle cap, and when the history restarts. The session
// drives a renderer through a small backend table, so the policy runs against the real renderer
// (gpsb_session_create) or against any other implementation of the same calls
// (gpsb_session_create_with_backend; the tests use a scripted fake on the CPU).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <new>

#include "gpsb200.h"

namespace {

constexpr uint32_t kSortMaxSplats = 8000000;  // lib.rs:84
constexpr double kSortSlowMs = 60.0;          // lib.rs:86
constexpr uint32_t kMaxPerSubmit = 4;         // gps.rs:19 (the reference's per-submit ensemble limit)

gpsb_status be_render(void* c, const gpsb_camera* cam, const gpsb_params* p, uint32_t seed, uint32_t n) {
    return gpsb_render_ensembles((gpsb_renderer*)c, cam, p, seed, n);
}
gpsb_status be_sorted(void* c, const gpsb_camera* cam, const gpsb_params* p, uint32_t n) {
    return gpsb_render_sorted((gpsb_renderer*)c, cam, p, n);
}
gpsb_status be_probe(void* c, const gpsb_camera* cam, const gpsb_params* p) {
    return gpsb_probe_demand((gpsb_renderer*)c, cam, p);
}
gpsb_status be_request(void* c) { return gpsb_request_stats((gpsb_renderer*)c); }
gpsb_status be_latest(void* c, gpsb_stats* s) { return gpsb_latest_stats((gpsb_renderer*)c, s); }
uint32_t be_issued(void* c) { return gpsb_stats_issued((gpsb_renderer*)c); }
uint32_t be_accumulated(void* c) { return gpsb_accumulated((gpsb_renderer*)c); }
uint32_t be_submitted(void* c) { return gpsb_submitted((gpsb_renderer*)c); }
gpsb_status be_reset_accum(void* c) { return gpsb_reset_accum((gpsb_renderer*)c); }
gpsb_status be_reset_stats(void* c) { return gpsb_reset_stats((gpsb_renderer*)c); }
uint32_t be_count(void* c) { return gpsb_gaussian_count((gpsb_renderer*)c); }

bool same_camera(const gpsb_camera& a, const gpsb_camera& b) { return memcmp(&a, &b, sizeof a) == 0; }

}  // namespace

struct gpsb_session {
    gpsb_session_backend be{};
    void* ctx = nullptr;
    gpsb_params params{};
    gpsb_camera cam{};
    bool have_cam = false;
    uint32_t seed = 1, next_seed = 1, per_frame = 1, target = 256;
    bool lod_adaptive = false;
    double lod_target_ms = 33.3, last_input_ms = -INFINITY, last_frame_ms = 0.0, ema_ms = 16.7;
    uint32_t effective_per_frame = 1, lod_n = 1, lod_quiet = 0;
    double point_budget = 0.0;
    float auto_density = 1.0f;
    uint32_t path_mode = 2;
    double demand_threshold = 30.0e6;
    bool sorted_active = false, sorted_ok = true;
    uint32_t probe_epoch = UINT32_MAX, decided_epoch = UINT32_MAX, probe_wait = 0, probe_issue = 0, slow_frames = 0;
    bool moving_prefers_gps = false;
    uint64_t last_demand = 0;
    uint32_t frames_since_reset = 0, ensemble_counter = 0, history_epoch = 0, moving_cap = 2048;
    bool lod_moving = false, dirty = true, needs_present = true;

    void invalidate() { dirty = true; }
    gpsb_params effective_params() const {
        gpsb_params p = params;
        p.density_scale *= auto_density;
        return p;
    }
};

extern "C" {

gpsb_status gpsb_session_create_with_backend(const gpsb_session_backend* be, void* ctx, gpsb_session** out) {
    if (!be || !out || !be->render_ensembles || !be->render_sorted || !be->probe_demand || !be->request_stats ||
        !be->latest_stats || !be->stats_issued || !be->accumulated || !be->submitted || !be->reset_accum ||
        !be->reset_stats || !be->gaussian_count)
        return GPSB_ERR_INVALID_ARGUMENT;
    gpsb_session* s = new (std::nothrow) gpsb_session();
    if (!s) return GPSB_ERR_OUT_OF_MEMORY;
    s->be = *be;
    s->ctx = ctx;
    gpsb_params_default(&s->params);
    *out = s;
    return GPSB_OK;
}

gpsb_status gpsb_session_create(gpsb_renderer* r, gpsb_session** out) {
    if (!r) return GPSB_ERR_INVALID_ARGUMENT;
    static const gpsb_session_backend real = {be_render, be_sorted,      be_probe,   be_request,
                                              be_latest, be_issued,      be_accumulated, be_submitted,
                                              be_reset_accum, be_reset_stats, be_count};
    return gpsb_session_create_with_backend(&real, r, out);
}

void gpsb_session_destroy(gpsb_session* s) { delete s; }

// Viewer::set_params / configure (lib.rs:325-350): parameters, ensembles per tick and target.
gpsb_status gpsb_session_configure(gpsb_session* s, const gpsb_params* p, uint32_t per_frame, uint32_t target) {
    if (!s || !p) return GPSB_ERR_INVALID_ARGUMENT;
    s->params = *p;
    s->params.density_scale = std::min(std::max(p->density_scale, 0.01f), 100.0f);
    s->params.max_points_per_splat = std::max(p->max_points_per_splat, 1u);
    s->per_frame = std::min(std::max(per_frame, 1u), kMaxPerSubmit);
    s->target = std::max(target, 1u);
    s->invalidate();
    return GPSB_OK;
}

// set_lod (lib.rs:437-443)
gpsb_status gpsb_session_set_lod(gpsb_session* s, int adaptive, double target_ms, uint32_t moving_cap) {
    if (!s) return GPSB_ERR_INVALID_ARGUMENT;
    s->lod_adaptive = adaptive != 0;
    s->lod_target_ms = std::min(std::max(target_ms, 8.0), 200.0);
    s->moving_cap = std::min(std::max(moving_cap, 64u), 1u << 24);
    s->invalidate();
    return GPSB_OK;
}

// set_point_budget (lib.rs:448-455)
gpsb_status gpsb_session_set_point_budget(gpsb_session* s, double millions) {
    if (!s) return GPSB_ERR_INVALID_ARGUMENT;
    double b = isfinite(millions) ? std::max(millions, 0.0) * 1.0e6 : 0.0;
    if (b != s->point_budget) {
        s->point_budget = b;
        s->auto_density = 1.0f;
        s->invalidate();
    }
    return GPSB_OK;
}

// set_render_path (lib.rs:461-473): 0 GPS particles, 1 sorted, 2 auto
gpsb_status gpsb_session_set_render_path(gpsb_session* s, uint32_t mode, double demand_threshold_millions) {
    if (!s) return GPSB_ERR_INVALID_ARGUMENT;
    mode = std::min(mode, 2u);
    double thr = isfinite(demand_threshold_millions)
                     ? std::min(std::max(demand_threshold_millions, 0.1), 100000.0) * 1.0e6
                     : 30.0e6;
    if (mode != s->path_mode || thr != s->demand_threshold) {
        s->path_mode = mode;
        s->demand_threshold = thr;
        s->sorted_ok = true;
        s->moving_prefers_gps = false;
        s->slow_frames = 0;
        s->decided_epoch = UINT32_MAX;
        s->invalidate();
    }
    return GPSB_OK;
}

// The camera of the next ticks; a different camera restarts the history. `user_input` != 0 marks
// it as interactive motion (orbit / pan / zoom, lib.rs:485-507), which drives the adaptive LOD.
gpsb_status gpsb_session_set_camera(gpsb_session* s, const gpsb_camera* cam, int user_input) {
    if (!s || !cam) return GPSB_ERR_INVALID_ARGUMENT;
    if (user_input) s->last_input_ms = s->last_frame_ms;
    if (!s->have_cam || !same_camera(s->cam, *cam)) {
        s->cam = *cam;
        s->have_cam = true;
        s->invalidate();
    }
    return GPSB_OK;
}

// reset (lib.rs:510-512)
gpsb_status gpsb_session_reset(gpsb_session* s) {
    if (!s) return GPSB_ERR_INVALID_ARGUMENT;
    s->invalidate();
    return GPSB_OK;
}

// One tick (Viewer::frame, lib.rs:523-697 without the surface): *presented = 1 when the
// accumulation changed and would be composited.
gpsb_status gpsb_session_frame(gpsb_session* s, double now_ms, int* presented) {
    if (!s || !s->have_cam) return GPSB_ERR_STATE;
    const gpsb_session_backend& be = s->be;
    void* c = s->ctx;
    double dt = s->last_frame_ms > 0.0 ? std::min(std::max(now_ms - s->last_frame_ms, 1.0), 500.0) : 16.7;
    s->last_frame_ms = now_ms;
    s->ema_ms += 0.1 * (dt - s->ema_ms);
    bool moving = s->lod_adaptive && now_ms - s->last_input_ms < 250.0;
    if (moving != s->lod_moving) {
        s->lod_moving = moving;
        s->dirty = true;  // the particle cap changes, so the history restarts
    }
    gpsb_status st;
    if (s->dirty) {
        if ((st = be.reset_accum(c)) != GPSB_OK) return st;
        if ((st = be.reset_stats(c)) != GPSB_OK) return st;
        s->history_epoch += 1;
        s->frames_since_reset = 0;
        s->next_seed = s->seed;
        s->dirty = false;
        s->needs_present = true;
    }
    if (be.submitted(c) <= s->target + 8) be.request_stats(c);
    const uint32_t acc = be.accumulated(c);
    if (s->frames_since_reset != UINT32_MAX) s->frames_since_reset += 1;
    gpsb_stats ls;
    memset(&ls, 0, sizeof ls);
    be.latest_stats(c, &ls);
    // point budget: demand of the current history window at density factor 1 (lib.rs:543-557)
    if (s->point_budget > 0.0 && !s->lod_moving && s->frames_since_reset >= 8 && ls.ensembles >= 2) {
        double demand = (double)(ls.points + ls.dropped_points) / (double)ls.ensembles / (double)s->auto_density;
        if (demand > 0.0) {
            float want = (float)std::min(std::max(s->point_budget / demand, 0.1), 1.0);
            if (fabsf(logf(want / s->auto_density)) > 0.25f) {
                s->auto_density = want;
                s->invalidate();
            }
        }
    }
    // render path (lib.rs:559-629)
    const bool moving_now = now_ms - s->last_input_ms < 250.0;
    const uint32_t count = be.gaussian_count(c);
    const bool sorted_eligible = s->params.method == 0u && count > 0 && count <= kSortMaxSplats;
    bool wait_for_probe = false;
    if (s->path_mode == 0) {
        s->sorted_active = false;
    } else if (s->path_mode == 1) {
        s->sorted_active = sorted_eligible && s->sorted_ok;
    } else {
        if (!(sorted_eligible && s->sorted_ok) || (moving_now && s->moving_prefers_gps)) {
            s->sorted_active = false;
        } else if (!moving_now && s->decided_epoch != s->history_epoch) {
            gpsb_params p = s->effective_params();
            if (s->probe_epoch != s->history_epoch) {
                if (be.probe_demand(c, &s->cam, &p) == GPSB_OK) {
                    s->probe_epoch = s->history_epoch;
                    s->probe_wait = 0;
                    s->probe_issue = be.stats_issued(c);
                } else {
                    s->sorted_ok = false;
                    s->sorted_active = false;
                }
            }
            if (s->probe_epoch == s->history_epoch) {
                be.request_stats(c);
                s->probe_wait += 1;
                be.latest_stats(c, &ls);
                if (ls.issue > s->probe_issue) {
                    double demand = (double)ls.probe_demand;
                    s->last_demand = ls.probe_demand;
                    double keep = s->sorted_active ? 0.5 : 1.0;  // hysteresis
                    s->sorted_active = demand > keep * s->demand_threshold;
                    s->decided_epoch = s->history_epoch;
                } else {
                    wait_for_probe = true;
                }
            }
        }
    }
    if (s->sorted_active) {
        if (moving_now && s->path_mode == 2) {
            s->slow_frames = s->ema_ms > kSortSlowMs ? s->slow_frames + 1 : 0;
            if (s->slow_frames >= 20) {
                s->moving_prefers_gps = true;
                s->sorted_active = false;
                s->slow_frames = 0;
                s->invalidate();
            }
        }
    } else {
        s->slow_frames = 0;
    }
    const bool stalled = acc == 0 && be.submitted(c) >= 8;
    if (s->sorted_active && !wait_for_probe) {
        if (acc < s->target) {
            gpsb_params p = s->effective_params();
            if (be.render_sorted(c, &s->cam, &p, s->target) == GPSB_OK) {
                s->effective_per_frame = 0;
                s->ensemble_counter += 1;
                s->needs_present = true;
            } else {
                s->sorted_ok = false;
                s->sorted_active = false;
                s->invalidate();
            }
        }
    } else if (wait_for_probe) {
        // keep the previous picture while the demand probe's readback is pending
    } else if (acc < s->target && !stalled) {
        if (moving_now) {
            s->lod_n = 1;
            s->lod_quiet = 0;
        }
        uint32_t want;
        if (!s->lod_adaptive) {
            want = s->per_frame;
        } else if (moving_now) {
            want = 1;
        } else {
            s->lod_quiet += 1;
            if (s->ema_ms > s->lod_target_ms) {
                s->lod_n = std::max(s->lod_n > 0 ? s->lod_n - 1 : 0u, 1u);
                s->lod_quiet = 0;
            } else if (s->ema_ms < 0.6 * s->lod_target_ms && s->lod_quiet >= 30) {
                s->lod_n = std::min(s->lod_n + 1, kMaxPerSubmit);
                s->lod_quiet = 0;
            }
            want = s->lod_n;
        }
        s->effective_per_frame = want;
        const uint32_t n = std::min(want, s->target - acc);
        gpsb_params p = s->effective_params();
        if (s->lod_moving) p.max_points_per_splat = std::min(p.max_points_per_splat, s->moving_cap);
        if ((st = be.render_ensembles(c, &s->cam, &p, s->next_seed, n)) != GPSB_OK) return st;
        s->next_seed += n;
        s->ensemble_counter += n;
        s->needs_present = true;
    }
    if (presented) *presented = s->needs_present ? 1 : 0;
    s->needs_present = false;
    return GPSB_OK;
}

gpsb_status gpsb_session_read_state(const gpsb_session* s, gpsb_session_state* out) {
    if (!s || !out) return GPSB_ERR_INVALID_ARGUMENT;
    memset(out, 0, sizeof *out);
    out->sorted_active = s->sorted_active;
    out->sorted_ok = s->sorted_ok;
    out->moving_prefers_gps = s->moving_prefers_gps;
    out->lod_moving = s->lod_moving;
    out->effective_per_frame = s->effective_per_frame;
    out->lod_n = s->lod_n;
    out->auto_density = s->auto_density;
    out->history_epoch = s->history_epoch;
    out->frames_since_reset = s->frames_since_reset;
    out->next_seed = s->next_seed;
    out->ensemble_counter = s->ensemble_counter;
    out->slow_frames = s->slow_frames;
    out->last_demand = s->last_demand;
    out->ema_ms = s->ema_ms;
    return GPSB_OK;
}

}  // extern "C"
