// Host side of the renderer: the C ABI of include/gpsb200.h over the CUDA kernels.
// Mirrors GpsRenderer (crates/gps-render/src/gps.rs) and SortedPath (sorted.rs): ownership,
// validation, error messages, history/statistics semantics. All GPU work of one renderer runs
// on one stream; render calls enqueue work and return (like queue.submit), readbacks wait.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <utility>
#include <string>
#include <vector>

#include "../../include/gpsb200.h"
#include "internal.h"
#include "sorted.h"

using namespace gpsb;

namespace gpsb {
void host_radius_lut(float* out);  // hostmath.cpp
}

static thread_local std::string g_last_error;

namespace gpsb {
void set_global_error(const char* msg) { g_last_error = msg; }
}

static const size_t kMaxSplats = 16000000;  // gps.rs:24

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    // Grows to at least `n` bytes; contents are not preserved.
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        release();
        size_t want = n < 256 ? 256 : n;
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            p = nullptr;
            return e;
        }
        bytes = want;
        return cudaSuccess;
    }
    template <class T> T* as() const { return (T*)p; }
};

struct gpsb_renderer {
    int device = 0;
    float* feat = nullptr;  // caller-owned denoiser feature sums (W*H*8 floats), or null
    cudaStream_t own = nullptr, stream = nullptr;
    uint32_t W = 0, H = 0, side = 1;
    uint32_t n = 0, sh_max_degree = 0, sh_stride = 0;
    double centroid[3] = {0, 0, 0};
    int sm_count = 148;
    // scene
    DevBuf splats, sh, lut;
    DevBuf spare[5];  // staging set of splats, sh, rec, cdesc, colour for the next scene
    // per camera
    DevBuf rec, cdesc, colour;
    // per frame
    DevBuf accum, stats, err;
    // per ensemble batch
    DevBuf sub, clist, lookback, etot, counters;
    uint32_t batch_cap = 0;
    uint32_t last_batch = 0;     // ensembles in the last batch rendered
    uint32_t last_seed = 0;      // seed of its first ensemble
    bool last_particle = false;  // whether it used the particle path
    // sorted path
    SortedState sorted;
    bool have_sorted = false;
    // composite
    DevBuf rgba8;
    // history / stats
    uint32_t accumulated = 0;
    unsigned long long* stats_pinned = nullptr;
    cudaEvent_t stats_event = nullptr;
    bool stats_pending = false;
    uint32_t stats_issued = 0;
    gpsb_stats latest{};
    std::string error;
    // profiling: CUDA-event pairs per stage, resolved at gpsb_profile_read
    bool prof_on = false;
    struct Pending { int stage; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    uint64_t launches[GPSB_STAGES] = {};
    double ms[GPSB_STAGES] = {};
    uint64_t total_launches = 0;
    // stand-alone primitives
    DevBuf prim_lookback, prim_counter;
    RadixScratch prim_sort;
    // launch-shape tuning
    uint32_t particle_items = 16, particle_blocks_per_sm = 5, ensemble_batch = 64;
    // footprint-subpixel Monte-Carlo mode (GPS)
    uint32_t fp_fixed = 1, fp_max = 4, fp_comp = 0;
    float fp_kappa = 0.0f;
    // PBVR fast decisions: 0 off, 1 on (default), 2 validate
    uint32_t fast_mode = 1;
    DevBuf dbg;
    // captured trajectory pipeline (gpsb_render_trajectory_graph) and the key of its work
    cudaGraphExec_t traj_exec = nullptr;
    std::vector<uint8_t> traj_key;
    uint64_t traj_launches = 0;
    uint64_t scene_gen = 0;
};

namespace gpsb {
// the renderer's stream and device, for the denoiser host code in this library
cudaStream_t renderer_stream(gpsb_renderer* r) { return r->stream; }
int renderer_device(gpsb_renderer* r) { return r->device; }
}  // namespace gpsb

// Brackets the kernels of one stage with CUDA events on the renderer's stream (when profiling)
// and counts the kernels launched.
struct StageScope {
    gpsb_renderer* r;
    int stage;
    cudaEvent_t a = nullptr;
    StageScope(gpsb_renderer* rr, int st) : r(rr), stage(st) {
        if (r->prof_on) {
            a = take();
            cudaEventRecord(a, r->stream);
        }
    }
    cudaEvent_t take() {
        if (!r->pool.empty()) {
            cudaEvent_t e = r->pool.back();
            r->pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void kernels(uint64_t n) {
        r->launches[stage] += n;
        r->total_launches += n;
    }
    ~StageScope() {
        if (r->prof_on && a) {
            cudaEvent_t b = take();
            cudaEventRecord(b, r->stream);
            r->pending.push_back({stage, a, b});
        }
    }
};

// ------------------------------------------------------------------------------ helpers
static gpsb_status fail(gpsb_renderer* r, gpsb_status s, const std::string& msg) {
    if (r) r->error = msg;
    g_last_error = msg;
    return s;
}
static gpsb_status cuda_fail(gpsb_renderer* r, cudaError_t e, const char* what) {
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    gpsb_status s = (e == cudaErrorMemoryAllocation) ? GPSB_ERR_OUT_OF_MEMORY : GPSB_ERR_CUDA;
    return fail(r, s, buf);
}
#define CK(r, call, what)                                    \
    do {                                                     \
        cudaError_t _e = (call);                             \
        if (_e != cudaSuccess) return cuda_fail(r, _e, what); \
    } while (0)

static uint32_t clamp_side(uint32_t s) { return std::max(1u, std::min(s, 4u)); }
static uint64_t sub_per_ensemble(const gpsb_renderer* r) { return (uint64_t)r->W * r->H * r->side * r->side; }

static FrameConst make_frame(const gpsb_renderer* r, const gpsb_camera& cam, const gpsb_params& p) {
    FrameConst f;
    memset(&f, 0, sizeof f);
    const double* R = cam.view_rot;
    for (int k = 0; k < 3; ++k) {
        f.rot0[k] = (float)R[k];
        f.rot1[k] = (float)R[3 + k];
        f.rot2[k] = (float)R[6 + k];
        f.pos[k] = (float)cam.view_pos[k];
    }
    f.low_pass = (float)cam.low_pass;
    f.jitter_sd = sqrtf(fmaxf(f.low_pass, 0.0f));
    double cx = cam.cx, cy = cam.cy;
    if (cam.cx == 0.0 && cam.cy == 0.0) {  // gps.rs:818
        cx = 0.5 * r->W;
        cy = 0.5 * r->H;
    }
    f.fx = (float)cam.focal_x;
    f.fy = (float)cam.focal_y;
    f.cx = (float)cx;
    f.cy = (float)cy;
    f.W = r->W;
    f.H = r->H;
    f.side = r->side;
    f.S = r->side * r->side;
    f.N = r->n;
    f.cap = std::max(p.max_points_per_splat, 1u);
    f.sh_stride = r->sh_stride;
    f.exact_radius = p.exact_radius ? 1u : 0u;
    f.density = p.density_scale;
    f.near_z = p.near_z;
    for (int k = 0; k < 3; ++k) f.bg[k] = p.background[k];
    f.method = p.method;
    f.calibration = p.pbvr.calibration;
    f.flags = (p.pbvr.radial_correction ? FLAG_RADIAL : 0u) | (p.pbvr.centre_depth ? FLAG_CENTRE : 0u) |
              (p.pbvr.low_pass_jitter ? FLAG_JITTER : 0u);
    f.sh_deg = std::min(p.sh_degree, r->sh_max_degree);
    f.base_k = p.pbvr.base_k;
    f.refl = p.pbvr.reference_pixel_length;
    double d[3] = {r->centroid[0] - cam.view_pos[0], r->centroid[1] - cam.view_pos[1], r->centroid[2] - cam.view_pos[2]};
    f.object_depth = (float)(R[6] * d[0] + R[7] * d[1] + R[8] * d[2]);
    f.fp_fixed = r->fp_fixed;
    f.fp_max = r->fp_max;
    f.fp_comp = r->fp_comp;
    f.fp_kappa = r->fp_kappa;
    f.fast_mode = r->fast_mode;
    return f;
}

static gpsb_status check_params(gpsb_renderer* r, const gpsb_camera* cam, const gpsb_params* p) {
    if (!cam || !p) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null camera or params");
    if (clamp_side(p->spp_side) != r->side)
        return fail(r, GPSB_ERR_INVALID_ARGUMENT, "params.spp_side differs from the renderer's; call resize() first");
    if (p->method > 4u) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "unknown method index");
    if (p->pbvr.calibration > 3u) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "unknown calibration level");
    return GPSB_OK;
}

static gpsb_status alloc_frame(gpsb_renderer* r) {
    uint64_t P = (uint64_t)r->W * r->H;
    CK(r, r->accum.ensure(P * 16), "accum buffer");
    CK(r, cudaMemsetAsync(r->accum.p, 0, P * 16, r->stream), "clear accum");
    r->batch_cap = 0;  // per-ensemble buffers depend on the resolution
    r->have_sorted = false;
    return GPSB_OK;
}

// Per-ensemble buffers for E ensembles of the current scene and resolution.
static gpsb_status ensure_batch(gpsb_renderer* r, uint32_t E) {
    if (E <= r->batch_cap) return GPSB_OK;
    uint64_t PS = sub_per_ensemble(r);
    uint32_t tiles = (r->n + kScanTile - 1) / kScanTile;
    CK(r, r->sub.ensure((size_t)E * PS * 8), "subpixel buffers");
    CK(r, r->clist.ensure((size_t)E * std::max(r->n, 1u) * 8), "particle list");
    CK(r, r->lookback.ensure((size_t)E * std::max(tiles, 1u) * 8), "scan lookback");
    CK(r, r->etot.ensure((size_t)E * sizeof(EnsTotal)), "ensemble totals");
    CK(r, r->counters.ensure(64), "counters");
    r->batch_cap = E;
    return GPSB_OK;
}

// Ensembles per batch: up to kDefaultBatch, fewer when the per-ensemble buffers would exceed
// a quarter of the free device memory.
static uint32_t pick_batch(gpsb_renderer* r, uint32_t count) {
    uint32_t want = std::min(count, r->ensemble_batch);
    if (want <= r->batch_cap) return want;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    uint64_t per = sub_per_ensemble(r) * 8 + (uint64_t)std::max(r->n, 1u) * 8 + 4096;
    uint64_t budget = (free_b + (uint64_t)r->sub.bytes + r->clist.bytes) / 4;
    uint64_t fit = per ? budget / per : want;
    if (fit < 1) fit = 1;
    return (uint32_t)std::min<uint64_t>(want, fit);
}

static gpsb_status geometry(gpsb_renderer* r, const FrameConst& f) {
    if (r->n == 0) return GPSB_OK;
    StageScope sc(r, GPSB_STAGE_GEOMETRY);
    sc.kernels(1);
    launch_geometry(f, r->splats.as<float4>(), r->sh.as<float>(), r->lut.as<float>(), r->rec.as<float4>(),
                    r->cdesc.as<uint2>(), r->colour.as<float4>(), r->stream);
    CK(r, cudaGetLastError(), "geometry kernel");
    return GPSB_OK;
}

// One batch of E ensembles (seeds first_seed..) of the current camera into `accum`.
static gpsb_status render_batch(gpsb_renderer* r, const FrameConst& f, bool particles, uint32_t first_seed, uint32_t E,
                                float4* accum) {
    uint64_t PS = sub_per_ensemble(r);
    ull_t* stats = r->stats.as<ull_t>();
    {
        StageScope sc(r, GPSB_STAGE_CLEAR);
        sc.kernels(1);
        CK(r, cudaMemsetAsync(r->sub.p, 0xFF, (size_t)E * PS * 8, r->stream), "clear subpixels");
        launch_add_stat(stats, ST_ENSEMBLES, E, r->stream);
    }
    uint32_t* cnt = r->counters.as<uint32_t>();
    if (particles) {
        {
            StageScope sc(r, GPSB_STAGE_COUNT_SCAN);
            sc.kernels(1);
            launch_count_scan(f, r->cdesc.as<uint2>(), first_seed, E, r->lookback.as<uint64_t>(), cnt,
                              r->clist.as<uint2>(), r->etot.as<EnsTotal>(), stats, r->err.as<uint32_t>(), r->stream);
            CK(r, cudaGetLastError(), "count/scan kernel");
        }
        {
            StageScope sc(r, GPSB_STAGE_PARTICLES);
            sc.kernels(1);
            launch_particles(f, r->rec.as<float4>(), r->lut.as<float>(), r->clist.as<uint2>(), r->etot.as<EnsTotal>(),
                             first_seed, E, r->sub.as<ull_t>(), cnt + 1, stats,
                             r->sm_count * (int)r->particle_blocks_per_sm, (int)r->particle_items, r->stream);
            CK(r, cudaGetLastError(), "particle kernel");
        }
    } else {
        StageScope sc(r, GPSB_STAGE_PRIMITIVE);
        sc.kernels(1);
        launch_primitive(f, r->rec.as<float4>(), r->cdesc.as<uint2>(), r->lut.as<float>(), first_seed, E,
                         r->sub.as<ull_t>(), r->etot.as<EnsTotal>(), stats, r->stream);
        CK(r, cudaGetLastError(), "primitive kernel");
    }
    {
        StageScope sc(r, GPSB_STAGE_RESOLVE);
        sc.kernels(1);
        launch_resolve(f, r->sub.as<ull_t>(), r->etot.as<EnsTotal>(), r->colour.as<float4>(), E, accum, stats,
                       r->stream);
        CK(r, cudaGetLastError(), "resolve kernel");
        if (r->feat) {
            sc.kernels(1);
            launch_features(f, r->sub.as<ull_t>(), r->etot.as<EnsTotal>(), r->colour.as<float4>(), E, r->feat,
                            r->stream);
            CK(r, cudaGetLastError(), "feature kernel");
        }
    }
    r->last_batch = E;
    r->last_seed = first_seed;
    r->last_particle = particles;
    return GPSB_OK;
}

static gpsb_status render_camera(gpsb_renderer* r, const gpsb_camera* cam, const gpsb_params* p, uint32_t first_seed,
                                 uint32_t count, float4* accum) {
    FrameConst f = make_frame(r, *cam, *p);
    bool particles = (p->path == GPSB_PATH_PARTICLE || p->method != GPSB_METHOD_GPS) && r->n > 0;
    gpsb_status s = geometry(r, f);
    if (s != GPSB_OK) return s;
    uint32_t B = pick_batch(r, count);
    s = ensure_batch(r, B);
    if (s != GPSB_OK) return s;
    for (uint32_t done = 0; done < count;) {
        uint32_t E = std::min(B, count - done);
        s = render_batch(r, f, particles, first_seed + done, E, accum);
        if (s != GPSB_OK) return s;
        done += E;
    }
    return GPSB_OK;
}

static void to_stats(const unsigned long long* w, gpsb_stats* out, uint32_t issue) {
    out->points = w[ST_POINTS];
    out->truncated_splats = w[ST_TRUNCATED];
    out->dropped_points = w[ST_DROPPED];
    out->visible_splats = w[ST_VISIBLE];
    out->orphan_subpixels = w[ST_ORPHAN];
    out->candidates = w[ST_CANDIDATES];
    out->undercovered_splats = w[ST_UNDERCOVERED];
    out->skipped_ensembles = w[ST_SKIPPED];
    out->ensembles = w[ST_ENSEMBLES];
    out->probe_demand = w[ST_PROBE];
    out->issue = issue;
    out->_pad = 0;
    out->subpixel_writes = w[ST_WRITES];
    out->list_entries = w[ST_ENTRIES];
    out->particles = w[ST_PARTICLES];
}

static void poll_stats(gpsb_renderer* r) {
    if (r->stats_pending && cudaEventQuery(r->stats_event) == cudaSuccess) {
        to_stats(r->stats_pinned, &r->latest, r->stats_issued);
        r->stats_pending = false;
    }
}

static gpsb_status check_error_word(gpsb_renderer* r) {
    uint32_t e = 0;
    CK(r, cudaMemcpyAsync(&e, r->err.p, 4, cudaMemcpyDeviceToHost, r->stream), "error word");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    if (e) {
        cudaMemsetAsync(r->err.p, 0, 4, r->stream);
        char buf[160];
        snprintf(buf, sizeof buf, "a bounded device-side wait gave up (error word 0x%x); the affected ensembles were skipped", e);
        return fail(r, GPSB_ERR_TIMEOUT, buf);
    }
    return GPSB_OK;
}

// ============================================================================== C ABI
extern "C" {

void gpsb_params_default(gpsb_params* p) {
    if (!p) return;
    memset(p, 0, sizeof *p);
    p->spp_side = 2;
    p->density_scale = 1.0f;
    p->max_points_per_splat = 1u << 16;
    p->near_z = 0.05f;
    p->background[0] = 0.05f;
    p->background[1] = 0.05f;
    p->background[2] = 0.08f;
    p->exposure = 1.0f;
    p->srgb_output = 1;
    p->exact_radius = 0;
    p->sh_degree = 3;
    p->path = GPSB_PATH_PARTICLE;
    p->method = GPSB_METHOD_GPS;
    p->pbvr.calibration = GPSB_CAL_PER_SPLAT_FOOTPRINT;
    p->pbvr.radial_correction = 0;
    p->pbvr.centre_depth = 0;
    p->pbvr.low_pass_jitter = 1;
    p->pbvr.base_k = 512.0f;
    p->pbvr.reference_pixel_length = 0.01f;
}

const char* gpsb_version(void) { return "gpsb200 0.1 (sm_100a)"; }

const char* gpsb_last_error(const gpsb_renderer* r) { return r ? r->error.c_str() : g_last_error.c_str(); }

void gpsb_estimate_memory(uint32_t w, uint32_t h, uint32_t spp_side, size_t n, uint64_t* dw, uint64_t* acc, uint64_t* sp) {
    uint64_t sub = (uint64_t)w * h * (uint64_t)(spp_side * spp_side);
    if (dw) *dw = 8 * sub;
    if (acc) *acc = 16ull * w * h;
    if (sp) *sp = 164ull * n;
}

gpsb_status gpsb_create(int device, uint32_t width, uint32_t height, uint32_t spp_side, gpsb_renderer** out) {
    if (!out) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    if (width == 0 || height == 0) return fail(nullptr, GPSB_ERR_LIMIT, "width/height must be > 0");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(nullptr, GPSB_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
    gpsb_renderer* r = new gpsb_renderer();
    r->device = device;
    r->W = width;
    r->H = height;
    r->side = clamp_side(spp_side);
    r->sm_count = device_sm_count(device);
    gpsb_status s = GPSB_OK;
    do {
        if ((e = cudaStreamCreateWithFlags(&r->own, cudaStreamNonBlocking)) != cudaSuccess) { s = cuda_fail(r, e, "stream"); break; }
        r->stream = r->own;
        if ((e = cudaEventCreateWithFlags(&r->stats_event, cudaEventDisableTiming)) != cudaSuccess) { s = cuda_fail(r, e, "event"); break; }
        if ((e = cudaMallocHost(&r->stats_pinned, ST_WORDS * 8)) != cudaSuccess) { s = cuda_fail(r, e, "pinned stats"); break; }
        if ((e = r->stats.ensure(ST_WORDS * 8)) != cudaSuccess) { s = cuda_fail(r, e, "stats"); break; }
        if ((e = r->err.ensure(256)) != cudaSuccess) { s = cuda_fail(r, e, "error word"); break; }
        cudaMemsetAsync(r->stats.p, 0, ST_WORDS * 8, r->stream);
        cudaMemsetAsync(r->err.p, 0, 4, r->stream);
        std::vector<float> lut(65 * 129);
        host_radius_lut(lut.data());
        if ((e = r->lut.ensure(lut.size() * 4)) != cudaSuccess) { s = cuda_fail(r, e, "radius table"); break; }
        cudaMemcpyAsync(r->lut.p, lut.data(), lut.size() * 4, cudaMemcpyHostToDevice, r->stream);
        if ((s = alloc_frame(r)) != GPSB_OK) break;
        if ((e = cudaStreamSynchronize(r->stream)) != cudaSuccess) { s = cuda_fail(r, e, "init"); break; }
    } while (0);
    if (s != GPSB_OK) {
        g_last_error = r->error;
        gpsb_destroy(r);
        return s;
    }
    *out = r;
    return GPSB_OK;
}

void gpsb_destroy(gpsb_renderer* r) {
    if (!r) return;
    cudaSetDevice(r->device);
    if (r->stream) cudaStreamSynchronize(r->stream);
    DevBuf* bufs[] = {&r->splats, &r->sh, &r->lut, &r->rec, &r->cdesc, &r->colour, &r->accum, &r->stats, &r->err,
                      &r->sub, &r->clist, &r->lookback, &r->etot, &r->counters, &r->rgba8};
    for (DevBuf* b : bufs) b->release();
    for (DevBuf& b : r->spare) b.release();
    sorted_release(r->sorted);
    r->prim_lookback.release();
    r->prim_counter.release();
    r->dbg.release();
    radix_release(r->prim_sort);
    for (auto& pe : r->pending) {
        cudaEventDestroy(pe.a);
        cudaEventDestroy(pe.b);
    }
    for (cudaEvent_t e : r->pool) cudaEventDestroy(e);
    if (r->traj_exec) cudaGraphExecDestroy(r->traj_exec);
    if (r->stats_pinned) cudaFreeHost(r->stats_pinned);
    if (r->stats_event) cudaEventDestroy(r->stats_event);
    if (r->own) cudaStreamDestroy(r->own);
    delete r;
}

gpsb_status gpsb_set_footprint(gpsb_renderer* r, uint32_t footprint_subpixels, float adaptive_kappa,
                              uint32_t footprint_max, uint32_t compensate_blur) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    if (footprint_subpixels > 64 || footprint_max > 64 || !(adaptive_kappa >= 0.0f) || !isfinite(adaptive_kappa))
        return fail(r, GPSB_ERR_INVALID_ARGUMENT, "footprint sizes must be 0..64 and kappa finite and >= 0");
    r->fp_fixed = std::max(footprint_subpixels, 1u);
    r->fp_max = std::max(footprint_max, 1u);
    r->fp_comp = compensate_blur ? 1u : 0u;
    r->fp_kappa = adaptive_kappa;
    return GPSB_OK;
}

gpsb_status gpsb_set_fast_decisions(gpsb_renderer* r, uint32_t mode) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    if (mode > 2) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "fast decision mode must be 0 (off), 1 (on) or 2 (validate)");
    r->fast_mode = mode;
    return GPSB_OK;
}

gpsb_status gpsb_debug_fast_counts(gpsb_renderer* r, uint64_t* counts) {
    if (!r || !counts) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null renderer or output");
    cudaSetDevice(r->device);
    unsigned long long w[ST_WORDS];
    CK(r, cudaMemcpyAsync(w, r->stats.p, sizeof w, cudaMemcpyDeviceToHost, r->stream), "read stats");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    counts[0] = w[ST_FAST_EXACT];
    counts[1] = w[ST_FAST_MISMATCH];
    return check_error_word(r);
}

gpsb_status gpsb_debug_fast_bounds(gpsb_renderer* r, float* ratios) {
    if (!r || !ratios) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null renderer or output");
    cudaSetDevice(r->device);
    CK(r, r->dbg.ensure(64), "debug scratch");
    launch_fast_bounds((uint32_t*)r->dbg.p, r->stream);
    CK(r, cudaGetLastError(), "fast bounds launch");
    CK(r, cudaMemcpyAsync(ratios, r->dbg.p, 6 * sizeof(float), cudaMemcpyDeviceToHost, r->stream), "read ratios");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    return GPSB_OK;
}

gpsb_status gpsb_set_feature_accum(gpsb_renderer* r, float* feat_dev) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    r->feat = feat_dev;
    return GPSB_OK;
}

gpsb_status gpsb_set_stream(gpsb_renderer* r, void* s) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    cudaSetDevice(r->device);
    CK(r, cudaStreamSynchronize(r->stream), "synchronise old stream");
    r->stream = s ? (cudaStream_t)s : r->own;
    return GPSB_OK;
}

static gpsb_status set_scene(gpsb_renderer* r, const void* g, size_t n, const float* sh, size_t sh_len, uint32_t degree,
                             cudaMemcpyKind kind) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    cudaSetDevice(r->device);
    if (n > 0 && !g) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null splat pointer");
    // gps.rs:694-701
    if ((uint64_t)n >= 0xFFFFFFFFull / 4) return fail(r, GPSB_ERR_LIMIT, "too many Gaussians for one dispatch");
    if (n > kMaxSplats) {
        char buf[160];
        snprintf(buf, sizeof buf, "%zu Gaussians exceeds the current limit of %zu", n, kMaxSplats);
        return fail(r, GPSB_ERR_LIMIT, buf);
    }
    uint32_t deg = 0, stride = 0;
    if (sh && degree >= 1 && n > 0) {
        uint32_t d = std::min(degree, 3u);
        stride = (d + 1) * (d + 1) - 1;
        if ((uint64_t)sh_len != (uint64_t)n * 3 * stride) {
            char buf[200];
            snprintf(buf, sizeof buf, "SH data has %zu values, expected %llu for %zu splats at degree %u", sh_len,
                     (unsigned long long)n * 3 * stride, n, degree);
            return fail(r, GPSB_ERR_INVALID_ARGUMENT, buf);
        }
        deg = d;
    }
    // Stage into the spare set of scene buffers so a failure keeps the old scene (gps.rs:682); the
    // sets swap afterwards, so reloading a scene of the same size allocates nothing.
    DevBuf &ns = r->spare[0], &nsh = r->spare[1], &nrec = r->spare[2], &ncd = r->spare[3], &ncol = r->spare[4];
    cudaError_t e;
    if ((e = ns.ensure(std::max<size_t>(n, 1) * 64)) != cudaSuccess ||
        (e = nsh.ensure(deg ? (size_t)n * 3 * stride * 4 : 64)) != cudaSuccess ||
        (e = nrec.ensure(std::max<size_t>(n, 1) * kRecF4 * 16)) != cudaSuccess ||
        (e = ncd.ensure(std::max<size_t>(n, 1) * 8)) != cudaSuccess ||
        (e = ncol.ensure(std::max<size_t>(n, 1) * 16)) != cudaSuccess) {
        return cuda_fail(r, e, "scene buffers");
    }
    if (n) e = cudaMemcpyAsync(ns.p, g, n * 64, kind, r->stream);
    if (e == cudaSuccess && deg) e = cudaMemcpyAsync(nsh.p, sh, (size_t)n * 3 * stride * 4, kind, r->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "scene upload");
    // centroid of the positions (gps.rs:731-735), from a host copy
    double c[3] = {0, 0, 0};
    if (n) {
        std::vector<gpsb_gaussian> host;
        const gpsb_gaussian* hg = (const gpsb_gaussian*)g;
        if (kind != cudaMemcpyHostToDevice) {
            host.resize(n);
            if ((e = cudaMemcpy(host.data(), ns.p, n * 64, cudaMemcpyDeviceToHost)) != cudaSuccess)
                return cuda_fail(r, e, "centroid readback");
            hg = host.data();
        }
        for (size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) c[k] = c[k] + (double)hg[i].pos_opacity[k];
        for (int k = 0; k < 3; ++k) c[k] = c[k] / (double)n;
    }
    std::swap(r->splats, ns);
    std::swap(r->sh, nsh);
    std::swap(r->rec, nrec);
    std::swap(r->cdesc, ncd);
    std::swap(r->colour, ncol);
    r->n = (uint32_t)n;
    r->sh_max_degree = deg;
    r->sh_stride = stride;
    memcpy(r->centroid, c, sizeof c);
    r->batch_cap = 0;  // the per-ensemble buffers grow to the new scene on the next render
    r->have_sorted = false;
    r->scene_gen += 1;
    return gpsb_reset_accum(r);
}

gpsb_status gpsb_set_gaussians(gpsb_renderer* r, const gpsb_gaussian* g, size_t n) {
    return set_scene(r, g, n, nullptr, 0, 0, cudaMemcpyHostToDevice);
}
gpsb_status gpsb_set_gaussians_sh(gpsb_renderer* r, const gpsb_gaussian* g, size_t n, const float* sh, size_t sh_len,
                                  uint32_t degree) {
    return set_scene(r, g, n, sh, sh_len, degree, cudaMemcpyHostToDevice);
}
gpsb_status gpsb_set_gaussians_sh_device(gpsb_renderer* r, const void* g, size_t n, const void* sh, size_t sh_len,
                                         uint32_t degree) {
    return set_scene(r, g, n, (const float*)sh, sh_len, degree, cudaMemcpyDeviceToDevice);
}

gpsb_status gpsb_resize(gpsb_renderer* r, uint32_t w, uint32_t h, uint32_t spp_side) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    cudaSetDevice(r->device);
    spp_side = clamp_side(spp_side);
    if (w == r->W && h == r->H && spp_side == r->side) return GPSB_OK;
    if (w == 0 || h == 0) return fail(r, GPSB_ERR_LIMIT, "width/height must be > 0");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    r->W = w;
    r->H = h;
    r->side = spp_side;
    r->feat = nullptr;  // sized for the old frame
    r->sub.release();
    r->accum.release();
    gpsb_status s = alloc_frame(r);
    if (s != GPSB_OK) return s;
    return gpsb_reset_accum(r);
}

gpsb_status gpsb_reset_accum(gpsb_renderer* r) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    cudaSetDevice(r->device);
    CK(r, cudaMemsetAsync(r->accum.p, 0, (size_t)r->W * r->H * 16, r->stream), "clear accum");
    r->accumulated = 0;
    // the skip counter belongs to the history window (gps.rs:796-800)
    CK(r, cudaMemsetAsync(r->stats.as<unsigned long long>() + ST_SKIPPED, 0, 8, r->stream), "clear skip counter");
    r->latest.skipped_ensembles = 0;
    return GPSB_OK;
}

gpsb_status gpsb_reset_stats(gpsb_renderer* r) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    cudaSetDevice(r->device);
    CK(r, cudaMemsetAsync(r->stats.p, 0, ST_WORDS * 8, r->stream), "clear stats");
    uint32_t issue = r->latest.issue;
    memset(&r->latest, 0, sizeof r->latest);
    r->latest.issue = issue;
    return GPSB_OK;
}

gpsb_status gpsb_render_ensembles(gpsb_renderer* r, const gpsb_camera* cam, const gpsb_params* p, uint32_t first_seed,
                                  uint32_t count) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    if (count == 0) return GPSB_OK;
    cudaSetDevice(r->device);
    gpsb_status s = check_params(r, cam, p);
    if (s != GPSB_OK) return s;
    s = render_camera(r, cam, p, first_seed, count, r->accum.as<float4>());
    if (s != GPSB_OK) return s;
    r->accumulated += count;
    return GPSB_OK;
}

gpsb_status gpsb_render_trajectory(gpsb_renderer* r, const gpsb_camera* cams, uint32_t n_cams, const gpsb_params* p,
                                   uint32_t first_seed, uint32_t E, void* accum_out_dev) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    if (n_cams == 0 || E == 0) return GPSB_OK;
    if (!cams || !accum_out_dev) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null cameras or output");
    cudaSetDevice(r->device);
    size_t P = (size_t)r->W * r->H;
    for (uint32_t c = 0; c < n_cams; ++c) {
        gpsb_status s = check_params(r, &cams[c], p);
        if (s != GPSB_OK) return s;
        float4* out = (float4*)accum_out_dev + (size_t)c * P;
        CK(r, cudaMemsetAsync(out, 0, P * 16, r->stream), "clear trajectory accum");
        s = render_camera(r, &cams[c], p, first_seed, E, out);
        if (s != GPSB_OK) return s;
    }
    return GPSB_OK;
}

// The trajectory's whole pipeline (per camera: clear, geometry, and per ensemble batch the count
// + scan, the persistent particle kernel and the resolve) captured once into a CUDA graph and
// replayed: a repeat with the same cameras, parameters, seeds, output, scene, resolution and
// tuning launches the graph again without re-encoding; anything else re-captures.
gpsb_status gpsb_render_trajectory_graph(gpsb_renderer* r, const gpsb_camera* cams, uint32_t n_cams,
                                         const gpsb_params* p, uint32_t first_seed, uint32_t E, void* accum_out_dev) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    if (n_cams == 0 || E == 0) return GPSB_OK;
    if (!cams || !accum_out_dev || !p) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null cameras, parameters or output");
    if (r->stream == nullptr) return fail(r, GPSB_ERR_STATE, "graph capture needs a non-default stream");
    if (r->prof_on) return fail(r, GPSB_ERR_STATE, "stage profiling is on; use gpsb_render_trajectory");
    if (r->feat) return fail(r, GPSB_ERR_STATE, "feature sums are on; use gpsb_render_trajectory");
    cudaSetDevice(r->device);
    for (uint32_t c = 0; c < n_cams; ++c) {
        gpsb_status s = check_params(r, &cams[c], p);
        if (s != GPSB_OK) return s;
    }
    // key of the captured work
    std::vector<uint8_t> key;
    auto put = [&](const void* d, size_t n) { key.insert(key.end(), (const uint8_t*)d, (const uint8_t*)d + n); };
    put(cams, sizeof(gpsb_camera) * n_cams);
    put(p, sizeof *p);
    uint32_t kappa_bits;
    memcpy(&kappa_bits, &r->fp_kappa, 4);
    uint64_t misc[] = {first_seed, E, (uint64_t)(uintptr_t)accum_out_dev, r->scene_gen, r->W, r->H, r->side,
                       r->particle_items, r->particle_blocks_per_sm, r->ensemble_batch, (uint64_t)r->sorted.digit_bits,
                       (uint64_t)(uintptr_t)r->stream, r->fp_fixed, r->fp_max, r->fp_comp,
                       (uint64_t)kappa_bits, r->fast_mode};
    put(misc, sizeof misc);
    // the device buffers baked into the graph: a reallocation (bigger batch, new scene or frame
    // size) must re-capture, never replay stale pointers
    const void* bufs[] = {r->splats.p, r->sh.p, r->lut.p, r->rec.p, r->cdesc.p, r->colour.p, r->stats.p, r->err.p,
                          r->sub.p, r->clist.p, r->lookback.p, r->etot.p, r->counters.p};
    put(bufs, sizeof bufs);
    if (!r->traj_exec || key != r->traj_key) {
        if (r->traj_exec) {
            cudaGraphExecDestroy(r->traj_exec);
            r->traj_exec = nullptr;
        }
        // every buffer the pipeline uses exists before the capture (no allocation inside it)
        uint32_t B = pick_batch(r, E);
        gpsb_status s = ensure_batch(r, B);
        if (s != GPSB_OK) return s;
        CK(r, r->counters.ensure(64), "counters");
        // the buffers may have just been (re)allocated: key them as they are now
        const void* now[] = {r->splats.p, r->sh.p, r->lut.p, r->rec.p, r->cdesc.p, r->colour.p, r->stats.p, r->err.p,
                             r->sub.p, r->clist.p, r->lookback.p, r->etot.p, r->counters.p};
        key.resize(key.size() - sizeof now);
        put(now, sizeof now);
        cudaGraph_t g = nullptr;
        const uint64_t launches0 = r->total_launches;
        CK(r, cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        const size_t P = (size_t)r->W * r->H;
        gpsb_status st = GPSB_OK;
        for (uint32_t c = 0; c < n_cams && st == GPSB_OK; ++c) {
            float4* out = (float4*)accum_out_dev + (size_t)c * P;
            if (cudaMemsetAsync(out, 0, P * 16, r->stream) != cudaSuccess) st = GPSB_ERR_CUDA;
            if (st == GPSB_OK) st = render_camera(r, &cams[c], p, first_seed, E, out);
        }
        cudaError_t e = cudaStreamEndCapture(r->stream, &g);
        if (st != GPSB_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(r, e, "capture of the trajectory");
        e = cudaGraphInstantiate(&r->traj_exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            r->traj_exec = nullptr;
            return cuda_fail(r, e, "graph instantiation");
        }
        r->traj_key = key;
        r->traj_launches = r->total_launches - launches0;
        r->total_launches = launches0;
    }
    CK(r, cudaGraphLaunch(r->traj_exec, r->stream), "graph launch");
    r->total_launches += r->traj_launches;
    return GPSB_OK;
}

gpsb_status gpsb_render_sorted(gpsb_renderer* r, const gpsb_camera* cam, const gpsb_params* p, uint32_t as_ensembles) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    cudaSetDevice(r->device);
    if (r->n == 0) return fail(r, GPSB_ERR_STATE, "empty scene");
    gpsb_status s = check_params(r, cam, p);
    if (s != GPSB_OK) return s;
    gpsb_params q = *p;
    q.method = GPSB_METHOD_GPS;  // gps.rs:935
    FrameConst f = make_frame(r, *cam, q);
    std::string msg;
    cudaError_t e;
    {
        StageScope sc(r, GPSB_STAGE_SORTED);
        sc.kernels(10);
        e = sorted_render(r->sorted, f, r->splats.as<float4>(), r->sh.as<float>(), r->accum.as<float4>(),
                          r->stats.as<unsigned long long>(), r->err.as<uint32_t>(), r->sm_count, true, r->stream, &msg);
    }
    if (e != cudaSuccess) return cuda_fail(r, e, msg.c_str());
    r->have_sorted = true;
    r->accumulated = std::max(as_ensembles, 1u);
    return GPSB_OK;
}

gpsb_status gpsb_probe_demand(gpsb_renderer* r, const gpsb_camera* cam, const gpsb_params* p) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    cudaSetDevice(r->device);
    if (r->n == 0) return fail(r, GPSB_ERR_STATE, "empty scene");
    if (!cam || !p) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null camera or params");
    FrameConst f = make_frame(r, *cam, *p);
    std::string msg;
    cudaError_t e;
    {
        StageScope sc(r, GPSB_STAGE_SORTED);
        sc.kernels(1);
        e = sorted_render(r->sorted, f, r->splats.as<float4>(), r->sh.as<float>(), r->accum.as<float4>(),
                          r->stats.as<unsigned long long>(), r->err.as<uint32_t>(), r->sm_count, false, r->stream, &msg);
    }
    if (e != cudaSuccess) return cuda_fail(r, e, msg.c_str());
    return GPSB_OK;
}

gpsb_status gpsb_read_accum(gpsb_renderer* r, float* out) {
    if (!r || !out) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null renderer or output");
    cudaSetDevice(r->device);
    CK(r, cudaMemcpyAsync(out, r->accum.p, (size_t)r->W * r->H * 16, cudaMemcpyDeviceToHost, r->stream), "read accum");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    return check_error_word(r);
}

gpsb_status gpsb_accum_device_ptr(gpsb_renderer* r, void** out) {
    if (!r || !out) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null renderer or output");
    *out = r->accum.p;
    return GPSB_OK;
}

gpsb_status gpsb_read_stats(gpsb_renderer* r, gpsb_stats* out) {
    if (!r || !out) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null renderer or output");
    cudaSetDevice(r->device);
    unsigned long long w[ST_WORDS];
    CK(r, cudaMemcpyAsync(w, r->stats.p, sizeof w, cudaMemcpyDeviceToHost, r->stream), "read stats");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    to_stats(w, out, 0);
    return check_error_word(r);
}

gpsb_status gpsb_request_stats(gpsb_renderer* r) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    cudaSetDevice(r->device);
    poll_stats(r);
    if (r->stats_pending) return GPSB_OK;  // one readback in flight (gps.rs:1006-1008)
    CK(r, cudaMemcpyAsync(r->stats_pinned, r->stats.p, ST_WORDS * 8, cudaMemcpyDeviceToHost, r->stream), "request stats");
    CK(r, cudaEventRecord(r->stats_event, r->stream), "stats event");
    r->stats_issued += 1;
    r->stats_pending = true;
    return GPSB_OK;
}

gpsb_status gpsb_latest_stats(gpsb_renderer* r, gpsb_stats* out) {
    if (!r || !out) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null renderer or output");
    poll_stats(r);
    *out = r->latest;
    return GPSB_OK;
}

uint32_t gpsb_stats_issued(const gpsb_renderer* r) { return r ? r->stats_issued : 0; }

gpsb_status gpsb_read_sorted(gpsb_renderer* r, uint32_t* keys, uint32_t* vals) {
    if (!r || !keys || !vals) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null argument");
    if (!r->have_sorted) return fail(r, GPSB_ERR_STATE, "no sorted render since the last scene/resize");
    cudaSetDevice(r->device);
    cudaError_t e = sorted_read(r->sorted, keys, vals, r->n, r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "read sorted");
    return GPSB_OK;
}

uint32_t gpsb_accumulated(gpsb_renderer* r) {
    if (!r) return 0;
    poll_stats(r);
    uint64_t sk = std::min<uint64_t>(r->latest.skipped_ensembles, 0xFFFFFFFFull);
    return r->accumulated > sk ? r->accumulated - (uint32_t)sk : 0u;
}
uint32_t gpsb_submitted(const gpsb_renderer* r) { return r ? r->accumulated : 0; }

gpsb_status gpsb_sync(gpsb_renderer* r) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    cudaSetDevice(r->device);
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    return check_error_word(r);
}

gpsb_status gpsb_composite_rgba8(gpsb_renderer* r, const gpsb_params* p, uint32_t out_w, uint32_t out_h, uint8_t* out) {
    if (!r || !p || !out) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null argument");
    if (out_w == 0 || out_h == 0) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "empty composite target");
    cudaSetDevice(r->device);
    size_t bytes = (size_t)out_w * out_h * 4;
    CK(r, r->rgba8.ensure(bytes), "composite target");
    {
        StageScope sc(r, GPSB_STAGE_COMPOSITE);
        sc.kernels(1);
        launch_composite(r->accum.as<float4>(), r->W, r->H, p->exposure, p->srgb_output ? 1u : 0u, out_w, out_h,
                         r->rgba8.as<uchar4>(), r->stream);
    }
    CK(r, cudaGetLastError(), "composite kernel");
    CK(r, cudaMemcpyAsync(out, r->rgba8.p, bytes, cudaMemcpyDeviceToHost, r->stream), "read composite");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    return GPSB_OK;
}

void gpsb_size(const gpsb_renderer* r, uint32_t* w, uint32_t* h, uint32_t* s) {
    if (!r) return;
    if (w) *w = r->W;
    if (h) *h = r->H;
    if (s) *s = r->side;
}
uint32_t gpsb_gaussian_count(const gpsb_renderer* r) { return r ? r->n : 0; }
uint32_t gpsb_sh_max_degree(const gpsb_renderer* r) { return r ? r->sh_max_degree : 0; }
uint64_t gpsb_sh_bytes(const gpsb_renderer* r) { return r ? (uint64_t)r->n * 3 * r->sh_stride * 4 : 0; }

gpsb_status gpsb_debug_read_counts(gpsb_renderer* r, uint32_t slot, uint32_t* counts) {
    if (!r || !counts) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null argument");
    if (!r->last_particle || slot >= r->last_batch) return fail(r, GPSB_ERR_STATE, "slot not in the last particle-path batch");
    cudaSetDevice(r->device);
    EnsTotal t;
    CK(r, cudaMemcpyAsync(&t, r->etot.as<EnsTotal>() + slot, sizeof t, cudaMemcpyDeviceToHost, r->stream), "read totals");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    std::vector<uint2> L(t.nonzero);
    if (t.nonzero)
        CK(r, cudaMemcpy(L.data(), r->clist.as<uint2>() + (size_t)slot * r->n, (size_t)t.nonzero * 8, cudaMemcpyDeviceToHost),
           "read list");
    memset(counts, 0, (size_t)r->n * 4);
    for (uint32_t j = 0; j < t.nonzero; ++j) {
        uint32_t end = j + 1 < t.nonzero ? L[j + 1].y : (uint32_t)t.particles;
        if (L[j].x < r->n) counts[L[j].x] = end - L[j].y;
    }
    return GPSB_OK;
}

gpsb_status gpsb_debug_particle_seeds(gpsb_renderer* r, uint32_t slot, uint64_t first_particle, uint32_t n,
                                      uint32_t* out) {
    if (!r || (n && !out)) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null argument");
    if (!r->last_particle || slot >= r->last_batch) return fail(r, GPSB_ERR_STATE, "slot not in the last particle-path batch");
    cudaSetDevice(r->device);
    EnsTotal t;
    CK(r, cudaMemcpyAsync(&t, r->etot.as<EnsTotal>() + slot, sizeof t, cudaMemcpyDeviceToHost, r->stream), "read totals");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    if (t.flags != 0u) return fail(r, GPSB_ERR_STATE, "the ensemble was skipped");
    if (first_particle > t.particles || n > t.particles - first_particle)
        return fail(r, GPSB_ERR_INVALID_ARGUMENT, "particle range beyond the ensemble's total");
    if (n == 0) return GPSB_OK;
    CK(r, r->dbg.ensure((size_t)n * 12), "debug buffer");
    launch_debug_seeds(r->clist.as<uint2>() + (size_t)slot * r->n, t.nonzero, first_particle, n, r->last_seed + slot,
                       r->dbg.as<uint32_t>(), r->stream);
    CK(r, cudaGetLastError(), "seed probe kernel");
    CK(r, cudaMemcpyAsync(out, r->dbg.p, (size_t)n * 12, cudaMemcpyDeviceToHost, r->stream), "read seeds");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    return GPSB_OK;
}

gpsb_status gpsb_debug_fmath(uint32_t which, const float* in_dev, float* out_dev, uint64_t n) {
    if ((which & 7u) > 4u || (which & ~15u) != 0u) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "which: 0..4, | 8");
    if (n && (!in_dev || !out_dev)) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null buffer");
    launch_debug_fmath(which, in_dev, out_dev, n, nullptr);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess) return fail(nullptr, GPSB_ERR_CUDA, std::string("fmath probe: ") + cudaGetErrorString(e));
    return GPSB_OK;
}

gpsb_status gpsb_debug_read_subpixels(gpsb_renderer* r, uint32_t slot, uint64_t* packed) {
    if (!r || !packed) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null argument");
    if (slot >= r->last_batch) return fail(r, GPSB_ERR_STATE, "slot not in the last batch");
    cudaSetDevice(r->device);
    uint64_t PS = sub_per_ensemble(r);
    CK(r, cudaMemcpyAsync(packed, r->sub.as<uint64_t>() + (size_t)slot * PS, PS * 8, cudaMemcpyDeviceToHost, r->stream),
       "read subpixels");
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    return GPSB_OK;
}

gpsb_status gpsb_scan_u32(gpsb_renderer* r, const uint32_t* in, uint32_t* out, uint32_t n, uint64_t* total) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    if (n && (!in || !out)) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null buffer");
    cudaSetDevice(r->device);
    CK(r, r->prim_lookback.ensure((size_t)std::max(scan_tiles(n), 1u) * 8), "scan lookback");
    CK(r, r->prim_counter.ensure(16), "scan counter");
    launch_scan_u32(in, out, n, r->prim_lookback.as<uint64_t>(), r->prim_counter.as<uint32_t>(), total,
                    r->err.as<uint32_t>(), r->stream);
    r->total_launches += 2;
    CK(r, cudaGetLastError(), "scan kernel");
    return GPSB_OK;
}

gpsb_status gpsb_sort_pairs(gpsb_renderer* r, uint32_t* ki, uint32_t* vi, uint32_t* ko, uint32_t* vo, uint32_t n,
                            uint32_t key_bits) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    if (key_bits < 1 || key_bits > 32) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "key_bits must be 1..32");
    if (n && (!ki || !vi || !ko || !vo)) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null buffer");
    if (n > (1u << 30)) return fail(r, GPSB_ERR_LIMIT, "at most 2^30 pairs");
    cudaSetDevice(r->device);
    cudaError_t e = radix_sort_pairs(r->prim_sort, ki, vi, ko, vo, n, (int)key_bits, r->sorted.digit_bits,
                                     r->err.as<uint32_t>(), r->stream);
    if (e != cudaSuccess) return cuda_fail(r, e, "radix sort");
    r->total_launches += 2 + (key_bits + r->sorted.digit_bits - 1) / r->sorted.digit_bits;
    return GPSB_OK;
}

gpsb_status gpsb_p0_sample(gpsb_renderer* r, uint32_t seed, uint32_t pixel_base, uint32_t pixels, uint32_t samples,
                           uint64_t* packed) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    if (samples && (!packed || pixels == 0)) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null buffer or no pixels");
    cudaSetDevice(r->device);
    launch_p0_sample(seed, pixel_base, pixels, samples, (unsigned long long*)packed, r->stream);
    r->total_launches += 1;
    CK(r, cudaGetLastError(), "p0 sample kernel");
    return GPSB_OK;
}

gpsb_status gpsb_set_tuning(gpsb_renderer* r, const gpsb_tuning* t) {
    if (!r || !t) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null argument");
    if (t->sort_digit_bits && t->sort_digit_bits != 4 && t->sort_digit_bits != 6 && t->sort_digit_bits != 8)
        return fail(r, GPSB_ERR_INVALID_ARGUMENT, "sort_digit_bits must be 4, 6 or 8");
    if (t->blend_tile_w || t->blend_tile_h) {
        bool ok = (t->blend_tile_w == 16 && t->blend_tile_h == 16) || (t->blend_tile_w == 32 && t->blend_tile_h == 8) ||
                  (t->blend_tile_w == 32 && t->blend_tile_h == 32);
        if (!ok) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "blend tiles must be 16x16, 32x8 or 32x32");
    }
    if (t->particle_items && t->particle_items != 8 && t->particle_items != 16 && t->particle_items != 24)
        return fail(r, GPSB_ERR_INVALID_ARGUMENT, "particle_items must be 8, 16 or 24");
    if (t->particle_blocks_per_sm > 32) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "particle_blocks_per_sm must be 1..32");
    if (t->ensemble_batch > 1024) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "ensemble_batch must be 1..1024");
    cudaSetDevice(r->device);
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    if (t->sort_digit_bits) r->sorted.digit_bits = (int)t->sort_digit_bits;
    if (t->blend_tile_w) {
        if (r->sorted.tw != t->blend_tile_w || r->sorted.th != t->blend_tile_h) r->have_sorted = false;
        r->sorted.tw = t->blend_tile_w;
        r->sorted.th = t->blend_tile_h;
    }
    if (t->particle_items) r->particle_items = t->particle_items;
    if (t->particle_blocks_per_sm) r->particle_blocks_per_sm = t->particle_blocks_per_sm;
    if (t->ensemble_batch) {
        r->ensemble_batch = t->ensemble_batch;
        r->batch_cap = 0;
        r->sub.release();
        r->clist.release();
        r->lookback.release();
        r->etot.release();
    }
    return GPSB_OK;
}

gpsb_status gpsb_get_tuning(const gpsb_renderer* r, gpsb_tuning* out) {
    if (!r || !out) return GPSB_ERR_INVALID_ARGUMENT;
    out->sort_digit_bits = (uint32_t)r->sorted.digit_bits;
    out->blend_tile_w = r->sorted.tw;
    out->blend_tile_h = r->sorted.th;
    out->particle_items = r->particle_items;
    out->particle_blocks_per_sm = r->particle_blocks_per_sm;
    out->ensemble_batch = r->ensemble_batch;
    return GPSB_OK;
}

static gpsb_status resolve_profile(gpsb_renderer* r) {
    if (r->pending.empty()) return GPSB_OK;
    CK(r, cudaStreamSynchronize(r->stream), "synchronise");
    for (auto& pe : r->pending) {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, pe.a, pe.b) == cudaSuccess) r->ms[pe.stage] += t;
        r->pool.push_back(pe.a);
        r->pool.push_back(pe.b);
    }
    r->pending.clear();
    return GPSB_OK;
}

gpsb_status gpsb_profile_enable(gpsb_renderer* r, int enable) {
    if (!r) return fail(nullptr, GPSB_ERR_INVALID_ARGUMENT, "null renderer");
    cudaSetDevice(r->device);
    gpsb_status s = resolve_profile(r);
    if (s != GPSB_OK) return s;
    r->prof_on = enable != 0;
    memset(r->launches, 0, sizeof r->launches);
    memset(r->ms, 0, sizeof r->ms);
    r->total_launches = 0;
    return GPSB_OK;
}

gpsb_status gpsb_profile_read(gpsb_renderer* r, gpsb_profile* out) {
    if (!r || !out) return fail(r, GPSB_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(r->device);
    gpsb_status s = resolve_profile(r);
    if (s != GPSB_OK) return s;
    for (int k = 0; k < GPSB_STAGES; ++k) {
        out->launches[k] = r->launches[k];
        out->ms[k] = r->ms[k];
    }
    out->total_launches = r->total_launches;
    return GPSB_OK;
}

uint32_t gpsb_debug_error_word(gpsb_renderer* r) {
    if (!r) return 0;
    uint32_t e = 0;
    cudaSetDevice(r->device);
    cudaMemcpyAsync(&e, r->err.p, 4, cudaMemcpyDeviceToHost, r->stream);
    cudaStreamSynchronize(r->stream);
    return e;
}

}  // extern "C"
