/* gpsb200: B200-native stochastic particle renderer for 3D Gaussian splats (GPS / PBVR).
 *
 * C ABI of the drop-in replacement for the wgpu renderer of gps-pbvr-web
 * (crates/gps-render/src/gps.rs, sorted.rs). Every entry point takes plain pointers and
 * sizes, returns a gpsb_status, and never aborts on user input; the message of the last
 * failure is available from gpsb_last_error(). One renderer is owned by one host thread and
 * runs its GPU work on its own CUDA stream (or a stream the caller supplies).
 *
 * Citations are file:line in the reference project.
 */
#ifndef GPSB200_H
#define GPSB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------ status */
typedef enum gpsb_status {
    GPSB_OK = 0,
    GPSB_ERR_INVALID_ARGUMENT = 1, /* bad size, null pointer, mismatched spp_side ... */
    GPSB_ERR_LIMIT = 2,            /* scene / resolution above a limit (gps.rs:572-590, 696-701) */
    GPSB_ERR_CUDA = 3,             /* a CUDA runtime call failed */
    GPSB_ERR_OUT_OF_MEMORY = 4,
    GPSB_ERR_TIMEOUT = 5,          /* a bounded device-side wait gave up (error word set) */
    GPSB_ERR_STATE = 6,            /* call not valid in the current state (e.g. no sorted render yet) */
    GPSB_ERR_PARSE = 7             /* PLY parse error (crates/gps-io/src/lib.rs:17-27) */
} gpsb_status;

/* ------------------------------------------------------------------------------ types */
/* One splat, 64 bytes, identical to GpuGaussian (gps.rs:26-38). */
typedef struct gpsb_gaussian {
    float pos_opacity[4]; /* xyz position, w = activated opacity */
    float log_scale[4];   /* xyz log of the per-axis standard deviation */
    float rot_wxyz[4];    /* (w, x, y, z), normalised by the renderer */
    float color[4];       /* xyz linear SH0 colour = f_dc * SH_C0 + 0.5 */
} gpsb_gaussian;

/* Pinhole camera of the oracle (crates/gps-core/src/oracle.rs:33-48): cam = view_rot *
 * (world - view_pos), +Z forward, image +Y down. A principal point of exactly (0, 0) means
 * the image centre (gps.rs:818). view_rot is row-major. */
typedef struct gpsb_camera {
    double view_rot[9];
    double view_pos[3];
    double focal_x, focal_y;
    double cx, cy;
    double low_pass; /* px^2 added to the projected covariance diagonal (default 0.3) */
} gpsb_camera;

/* Method indices (gps.rs:104-127). */
enum {
    GPSB_METHOD_GPS = 0,
    GPSB_METHOD_PROPORTIONAL = 1,
    GPSB_METHOD_EXTINCTION = 2,
    GPSB_METHOD_VIEW_CONDITIONED = 3,
    GPSB_METHOD_SCREEN_OCCUPANCY = 4
};
/* Calibration levels C0..C3 (gps.rs:144-165). */
enum {
    GPSB_CAL_NONE = 0,
    GPSB_CAL_OBJECT_ZOOM = 1,
    GPSB_CAL_PER_SPLAT_DEPTH = 2,
    GPSB_CAL_PER_SPLAT_FOOTPRINT = 3
};
/* RenderPath (gps.rs:93-100): the splat-parallel primitive path is the validation path. */
enum { GPSB_PATH_PRIMITIVE = 0, GPSB_PATH_PARTICLE = 1 };

/* PbvrParams (gps.rs:169-185). Booleans are 0/1. */
typedef struct gpsb_pbvr_params {
    uint32_t calibration;
    uint32_t radial_correction;
    uint32_t centre_depth;
    uint32_t low_pass_jitter;
    float base_k;
    float reference_pixel_length;
} gpsb_pbvr_params;

/* RenderParams (gps.rs:189-229). */
typedef struct gpsb_params {
    uint32_t spp_side;             /* subpixels per pixel = spp_side^2, 1..4 */
    float density_scale;
    uint32_t max_points_per_splat;
    float near_z;
    float background[3];
    float exposure;
    uint32_t srgb_output;
    uint32_t exact_radius;
    uint32_t sh_degree;
    uint32_t path;
    uint32_t method;
    gpsb_pbvr_params pbvr;
} gpsb_params;

/* GpuStats (gps.rs:231-272): cumulative since gpsb_reset_stats. */
typedef struct gpsb_stats {
    uint64_t points;
    uint64_t truncated_splats;
    uint64_t dropped_points;
    uint64_t visible_splats;
    uint64_t orphan_subpixels;
    uint64_t candidates;
    uint64_t undercovered_splats;
    uint64_t skipped_ensembles;
    uint64_t ensembles;
    uint64_t probe_demand;
    uint32_t issue;
    uint32_t _pad;
    /* no reference counterpart: particles written to an on-screen subpixel (the oracle's
     * RenderStats::subpixel_writes, crates/gps-core/src/oracle.rs:99-104) and entries of the
     * per-ensemble compact particle lists; they size the algorithmic bytes of the kernels */
    uint64_t subpixel_writes;
    uint64_t list_entries;
    /* no reference counterpart: particles generated (the per-ensemble totals of the scan, summed
     * over the ensembles that were not skipped), on screen or not */
    uint64_t particles;
} gpsb_stats;

/* Device-time profile of the renderer's kernels (no reference counterpart; the reference has
 * no GPU timestamps, gps.rs:888). Stages: */
enum {
    GPSB_STAGE_GEOMETRY = 0,
    GPSB_STAGE_COUNT_SCAN = 1,
    GPSB_STAGE_PARTICLES = 2,
    GPSB_STAGE_RESOLVE = 3,
    GPSB_STAGE_CLEAR = 4,
    GPSB_STAGE_PRIMITIVE = 5,
    GPSB_STAGE_SORTED = 6,
    GPSB_STAGE_COMPOSITE = 7,
    GPSB_STAGES = 8
};
typedef struct gpsb_profile {
    uint64_t launches[8];    /* kernels of this library launched per stage */
    double ms[8];            /* summed device time per stage (CUDA events on the renderer's stream) */
    uint64_t total_launches; /* kernels launched since gpsb_create or the last gpsb_profile_enable */
} gpsb_profile;

typedef struct gpsb_renderer gpsb_renderer;

/* --------------------------------------------------------------------- defaults / misc */
/* RenderParams::default() and PbvrParams::default() (gps.rs:181-228). */
void gpsb_params_default(gpsb_params* out);
/* Library version string. */
const char* gpsb_version(void);
/* Message of the last failure of `r` (or of the last gpsb_create / free function when r is NULL). */
const char* gpsb_last_error(const gpsb_renderer* r);

/* OracleCamera::look_at (crates/gps-core/src/oracle.rs:53-70). fov_y in radians. */
gpsb_status gpsb_camera_look_at(const double eye[3], const double target[3], const double up[3],
                                double fov_y, uint32_t w, uint32_t h, gpsb_camera* out);
/* OrbitCamera::to_camera (crates/gps-core/src/camera.rs:31-65). */
gpsb_status gpsb_orbit_camera(const double target[3], double distance, double yaw, double pitch,
                              const double up[3], double fov_y, uint32_t w, uint32_t h,
                              gpsb_camera* out);
/* OrbitCamera::robust_sphere (camera.rs:70-84) over xyz of n splats. */
gpsb_status gpsb_robust_sphere(const gpsb_gaussian* splats, size_t n, double centre[3], double* radius);

/* gps_core::radius_lut (crates/gps-core/src/lib.rs:624-636): 65 x 129 f32 table. */
gpsb_status gpsb_radius_lut(float* out_8385);

/* Estimated per-frame GPU bytes (gps.rs:288-291): depth+winner, accum, splats. */
void gpsb_estimate_memory(uint32_t w, uint32_t h, uint32_t spp_side, size_t n_splats,
                          uint64_t* depth_winner_bytes, uint64_t* accum_bytes, uint64_t* splat_bytes);

/* ------------------------------------------------------------------- construction */
/* GpsRenderer::new (gps.rs:380-570). spp_side is clamped to 1..4. device = CUDA ordinal. */
gpsb_status gpsb_create(int device, uint32_t width, uint32_t height, uint32_t spp_side,
                        gpsb_renderer** out);
/* Releases every GPU resource of `r` (Drop of GpsRenderer). NULL is a no-op. */
void gpsb_destroy(gpsb_renderer* r);
/* Run the renderer's work on an external cudaStream_t (NULL restores its own stream). */
gpsb_status gpsb_set_stream(gpsb_renderer* r, void* cuda_stream);
/* Footprint-subpixel Monte-Carlo mode of the GPS method (the reference has it only in its CPU
 * oracle: render_monte_carlo's MonteCarloOptions, crates/gps-core/src/oracle.rs:203-310,
 * lib.rs:412-433): each particle writes a footprint_subpixels x footprint_subpixels block of
 * subpixels (write_block) and the expected count is divided by its area; adaptive_kappa > 0
 * picks the footprint per splat as floor(kappa * smallest standard deviation in subpixels),
 * clamped to 1..footprint_max; compensate_blur shrinks the sampling covariance by the block's
 * blur. footprint_subpixels <= 1 with adaptive_kappa = 0 is the normal GPS renderer. */
gpsb_status gpsb_set_footprint(gpsb_renderer* r, uint32_t footprint_subpixels, float adaptive_kappa,
                              uint32_t footprint_max, uint32_t compensate_blur);
/* PBVR fast decisions (no counterpart in the reference, whose shader runs every particle through
 * the full path): 0 off; 1 on, where particles that bounded approximate maths proves are not
 * points or are points off screen skip the exact path, which leaves every output bit-identical;
 * 2 validate, where every particle runs the exact path and the fast answer is checked against it
 * (gpsb_debug_fast_counts). Default 1. */
gpsb_status gpsb_set_fast_decisions(gpsb_renderer* r, uint32_t mode);
/* Of the last frame: counts[0] = particles the fast decisions left to the exact path, counts[1] =
 * fast answers that disagreed with the exact path (mode 2; always 0 when the bounds hold). */
gpsb_status gpsb_debug_fast_counts(gpsb_renderer* r, uint64_t* counts);
/* Exhaustive check of the fast decisions' approximation constants over every input they can get:
 * ratios[0..5] = largest |approximation - exact| / bound of log (uniforms), log ([1e-6, 1)),
 * sin/cos, the Box-Muller radius, the radius' maximum, exp ([-128, 0]); each <= 1 when the bounds
 * hold. */
gpsb_status gpsb_debug_fast_bounds(gpsb_renderer* r, float* ratios);
/* Denoiser features (no counterpart in the reference, which has no denoiser): with feat_dev set
 * (device memory of the caller, width*height*8 floats, zeroed by the caller), every rendered
 * ensemble also adds, per pixel, (r^2, g^2, b^2, alpha, depth) of its resolved colour, covered
 * subpixel fraction and covered depth sum / subpixels to feat_dev[pixel*8 + 0..4]. NULL turns it
 * off; gpsb_resize turns it off. */
gpsb_status gpsb_set_feature_accum(gpsb_renderer* r, float* feat_dev);

/* ------------------------------------------------------------------- scene */
/* GpsRenderer::set_gaussians (gps.rs:683). Host pointer. On error the old scene stays. The new
 * scene is staged in a second set of scene buffers that then swaps with the current one, so the
 * renderer holds two scenes' worth of device memory after the first reload, and reloading a
 * scene no larger than one it held before allocates nothing. */
gpsb_status gpsb_set_gaussians(gpsb_renderer* r, const gpsb_gaussian* splats, size_t n);
/* GpsRenderer::set_gaussians_sh (gps.rs:689-740): sh_rest holds 3*((d+1)^2-1) floats per
 * splat, channel-major (R.., G.., B..); sh_len must equal n*3*((d+1)^2-1) when degree >= 1. */
gpsb_status gpsb_set_gaussians_sh(gpsb_renderer* r, const gpsb_gaussian* splats, size_t n,
                                  const float* sh_rest, size_t sh_len, uint32_t degree);
/* The same from device pointers (no host staging). */
gpsb_status gpsb_set_gaussians_sh_device(gpsb_renderer* r, const void* splats_dev, size_t n,
                                         const void* sh_rest_dev, size_t sh_len, uint32_t degree);

/* GpsRenderer::resize (gps.rs:781-789): reallocates per-frame buffers, resets history. */
gpsb_status gpsb_resize(gpsb_renderer* r, uint32_t width, uint32_t height, uint32_t spp_side);
/* reset_accum (gps.rs:792-801) also restarts the skipped-ensemble counter. */
gpsb_status gpsb_reset_accum(gpsb_renderer* r);
/* reset_stats (gps.rs:803-809). */
gpsb_status gpsb_reset_stats(gpsb_renderer* r);

/* ------------------------------------------------------------------- render */
/* GpsRenderer::render_ensembles (gps.rs:861-925): `count` independent ensembles with seeds
 * first_seed .. first_seed+count-1 accumulated into the history. The reference accepts at
 * most 4 per call (gps.rs:19); any count is accepted here and batched on the device. */
gpsb_status gpsb_render_ensembles(gpsb_renderer* r, const gpsb_camera* cam, const gpsb_params* p,
                                  uint32_t first_seed, uint32_t count);
/* Batched trajectory (no reference counterpart; the frame loop of gps-web renders one camera
 * at a time): for every camera c, ensembles first_seed .. first_seed+E-1 are accumulated into
 * a fresh accumulation written to accum_out_dev + c*W*H*4 floats (device pointer, RGB sum and
 * count like read_accum). The renderer's own history is not touched. */
gpsb_status gpsb_render_trajectory(gpsb_renderer* r, const gpsb_camera* cams, uint32_t n_cams,
                                   const gpsb_params* p, uint32_t first_seed,
                                   uint32_t ensembles_per_camera, void* accum_out_dev);
/* The same trajectory through one captured CUDA graph (no counterpart in the reference, which
 * encodes every pass per submit): the first call captures the whole pipeline of all cameras and
 * ensemble batches on the renderer's stream and launches it; a repeat with identical cameras,
 * parameters, seeds, output buffer, scene, frame size and tuning only relaunches the graph, any
 * change re-captures. Needs a non-default stream (the renderer's own, or gpsb_set_stream with a
 * created stream); refused while stage profiling or feature sums are on. */
gpsb_status gpsb_render_trajectory_graph(gpsb_renderer* r, const gpsb_camera* cams, uint32_t n_cams,
                                         const gpsb_params* p, uint32_t first_seed, uint32_t ensembles_per_camera,
                                         void* accum_out_dev);
/* render_sorted (gps.rs:930-944): depth-sorted alpha image written into the history with
 * count 1 and reported as `as_ensembles` accumulated ensembles. */
gpsb_status gpsb_render_sorted(gpsb_renderer* r, const gpsb_camera* cam, const gpsb_params* p,
                               uint32_t as_ensembles);
/* probe_demand (gps.rs:948-955): GPS particle demand of the view into stats.probe_demand. */
gpsb_status gpsb_probe_demand(gpsb_renderer* r, const gpsb_camera* cam, const gpsb_params* p);

/* ------------------------------------------------------------------- readback */
/* read_accum (gps.rs:989-993): W*H*4 floats (RGB sum, A = count). Host pointer. Synchronises. */
gpsb_status gpsb_read_accum(gpsb_renderer* r, float* rgba_host);
/* Device pointer of the accumulation buffer (valid until the next resize/destroy). */
gpsb_status gpsb_accum_device_ptr(gpsb_renderer* r, void** out);
/* read_stats (gps.rs:996-1000). Synchronises. */
gpsb_status gpsb_read_stats(gpsb_renderer* r, gpsb_stats* out);
/* request_stats / latest_stats / stats_issued (gps.rs:1005-1038): one readback in flight. */
gpsb_status gpsb_request_stats(gpsb_renderer* r);
gpsb_status gpsb_latest_stats(gpsb_renderer* r, gpsb_stats* out);
uint32_t gpsb_stats_issued(const gpsb_renderer* r);
/* read_sorted test hook (gps.rs:958-963): n keys and n values of the last sorted render. */
gpsb_status gpsb_read_sorted(gpsb_renderer* r, uint32_t* keys, uint32_t* vals);
/* accumulated() = submitted - skipped (gps.rs:675-677); submitted() (gps.rs:669-671). */
uint32_t gpsb_accumulated(gpsb_renderer* r);
uint32_t gpsb_submitted(const gpsb_renderer* r);
/* wait_idle (gps.rs:1055-1057). */
gpsb_status gpsb_sync(gpsb_renderer* r);
/* composite (gps.rs:967-986, shaders/gps_composite.wgsl) into a headless RGBA8 buffer of
 * out_w x out_h (bilinear up/down-sampling in linear space, exposure, optional sRGB OETF). */
gpsb_status gpsb_composite_rgba8(gpsb_renderer* r, const gpsb_params* p, uint32_t out_w,
                                 uint32_t out_h, uint8_t* out_host);

/* ------------------------------------------------------------------- queries */
void gpsb_size(const gpsb_renderer* r, uint32_t* w, uint32_t* h, uint32_t* spp_side);
uint32_t gpsb_gaussian_count(const gpsb_renderer* r);
uint32_t gpsb_sh_max_degree(const gpsb_renderer* r);
uint64_t gpsb_sh_bytes(const gpsb_renderer* r);

/* ------------------------------------------------------------------- test hooks */
/* Per-splat particle counts (after the cap) of ensemble `slot` of the last particle-path
 * render call (slot < min(count, batch)); n entries. Used by the bit-exact parity tests. */
gpsb_status gpsb_debug_read_counts(gpsb_renderer* r, uint32_t slot, uint32_t* counts);
/* Packed subpixel winners ((depth key << 32) | splat id, all ones = empty) of ensemble
 * `slot` of the last render call; W*H*spp entries. */
gpsb_status gpsb_debug_read_subpixels(gpsb_renderer* r, uint32_t slot, uint64_t* packed);
/* Device-side error word (bounded waits that gave up); 0 when healthy. */
uint32_t gpsb_debug_error_word(gpsb_renderer* r);
/* Stream seeds of particles first_particle .. first_particle + n - 1 of ensemble `slot` of the
 * last particle-path render call, as the particle kernel derives them: out[3 j .. 3 j + 2] =
 * (splat i, index k within the splat, particle_seed(i, k + 1, seed of the ensemble)), the splat
 * found in the compact list by the particle kernel's search (shaders/gps_splat.wgsl:63-68,
 * 667-680; crates/gps-core/src/lib.rs:450-465). Synchronous; host output of 3 n words. */
gpsb_status gpsb_debug_particle_seeds(gpsb_renderer* r, uint32_t slot, uint64_t first_particle, uint32_t n,
                                      uint32_t* out);
/* The shared exp/log/sin/cos evaluated on the current device exactly as the kernels evaluate
 * them: which 0 exp, 1 log, 2 sin, 3 cos, 4 log of a positive normal argument, tables in shared
 * memory (the particle kernel's form); which | 8 reads the global tables (the other kernels'
 * form). in_dev/out_dev: n floats of device memory. Synchronous (legacy default stream). */
gpsb_status gpsb_debug_fmath(uint32_t which, const float* in_dev, float* out_dev, uint64_t n);

/* Launch-shape tuning (no reference counterpart). Zero fields keep the current value.
 *   sort_digit_bits        radix digit width of the depth sort: 4, 6 or 8 (default 8)
 *   blend_tile_w/h         screen tiles of the sorted blend: 16x16 (default), 32x8 or 32x32
 *   particle_items         particles per thread per tile of the particle kernel: 8, 16 (default), 24
 *   particle_blocks_per_sm persistent grid of the particle kernel (default 5 per SM)
 *   ensemble_batch         most ensembles per device batch (default 64, at most 1024) */
typedef struct gpsb_tuning {
    uint32_t sort_digit_bits;
    uint32_t blend_tile_w, blend_tile_h;
    uint32_t particle_items;
    uint32_t particle_blocks_per_sm;
    uint32_t ensemble_batch;
} gpsb_tuning;
gpsb_status gpsb_set_tuning(gpsb_renderer* r, const gpsb_tuning* t);
gpsb_status gpsb_get_tuning(const gpsb_renderer* r, gpsb_tuning* out);

/* Stage timing: enable (1) or disable (0) CUDA-event timing of every stage; both reset the
 * profile. Launch counting is always on. */
gpsb_status gpsb_profile_enable(gpsb_renderer* r, int enable);
/* Reads the profile (synchronises the renderer's stream). */
gpsb_status gpsb_profile_read(gpsb_renderer* r, gpsb_profile* out);

/* ------------------------------------------------------------------- primitives */
/* Exclusive scan of n u32 counts (device pointers) on the renderer's stream: the single-pass
 * decoupled-lookback scan that replaces the hierarchical scan of shaders/gps_scan.wgsl (checked
 * by the reference at n in {1, 255, 256, 257, 65536, 300000, 1000003}, lib.rs:196-275). out may
 * equal in. The 64-bit total goes to *total_dev when it is not NULL. Enqueues and returns. */
gpsb_status gpsb_scan_u32(gpsb_renderer* r, const uint32_t* in_dev, uint32_t* out_dev, uint32_t n,
                          uint64_t* total_dev);
/* Stable ascending radix sort of n (key, value) pairs on the low key_bits bits, with the digit
 * width of gpsb_tuning (shaders/gps_sort.wgsl semantics). keys_in/vals_in are clobbered; scratch
 * belongs to the renderer. Enqueues and returns. */
gpsb_status gpsb_sort_pairs(gpsb_renderer* r, uint32_t* keys_in, uint32_t* vals_in, uint32_t* keys_out,
                            uint32_t* vals_out, uint32_t n, uint32_t key_bits);
/* Phase-0 winner-rule check (shaders/p0_sample.wgsl, lib.rs:99-192): `samples` synthetic samples
 * of ensemble `seed` written with one packed atomicMin into packed_dev[pixel_base .. +pixels)
 * (u64 (depth key << 32) | colour; initialise to all ones). Enqueues and returns. */
gpsb_status gpsb_p0_sample(gpsb_renderer* r, uint32_t seed, uint32_t pixel_base, uint32_t pixels,
                           uint32_t samples, uint64_t* packed_dev);

/* ------------------------------------------------------------------- sort without allocation */
/* No counterpart in the reference. Stable ascending LSD radix sort of n (key, value) pairs on
 * the low key_bits bits (1..32, keys must be below 2^key_bits), the onesweep kernels of the
 * depth-sorted path, for callers that cannot allocate device memory: a host that owns the whole
 * GPU memory budget through its own pool, or a real-time frame loop in which a cudaMalloc would
 * stall or is not allowed. It allocates nothing: all four pointers are device memory of the
 * caller; the sorted pairs are written to keys_out/vals_out and keys_in/vals_in are overwritten
 * (they are the ping-pong buffer). Its scratch is a fixed array inside this library (about
 * 1.35 MB, held by every GPU that loads the library until the process exits), which limits n to
 * 2,097,152 pairs; larger n returns GPSB_ERR_LIMIT. Each call whose stream is not being captured
 * looks the array's device address up (cudaGetSymbolAddress, with the call's device current), so
 * a device reset in between is harmless; a call made while its stream is being captured uses the
 * address of the last uncaptured call on that device, and without one it returns GPSB_ERR_STATE:
 * make the first call on a device before any stream capture. Work is enqueued on cuda_stream
 * (NULL = the legacy default stream) and the call returns without waiting. Every call shares the
 * one array, which keeps the last call's contents: each call clears what it needs, but calls that
 * overlap on the GPU (on different streams, or from several threads) race and give wrong results.
 * err_dev is a device word of the caller and must not be NULL: a bounded device-side wait that
 * gives up ORs a non-zero value into it (the sort's output is then not valid). Messages of failed
 * calls: gpsb_last_error(NULL). */
gpsb_status gpsb_sort_pairs_noalloc(uint32_t* keys_in, uint32_t* vals_in, uint32_t* keys_out,
                                    uint32_t* vals_out, uint32_t n, uint32_t key_bits,
                                    void* cuda_stream, uint32_t* err_dev);

/* ------------------------------------------------------------------- frame-loop session
 * The reference viewer's frame policy (crates/gps-web/src/lib.rs:437-697: Viewer::frame, set_lod,
 * set_point_budget, set_render_path), headless: per tick it restarts the history when the
 * camera, parameters or LOD state change, keeps the non-blocking statistics readback going,
 * adapts the point-budget density factor, picks GPS particles or the depth-sorted path (Auto:
 * demand probe of the still view, switch above the threshold with 0.5 hysteresis, hand motion
 * to particles when sorting is slow), and renders the manual or adaptive number of ensembles
 * (one while the camera moves, with the moving-camera particle cap). Half-resolution rendering
 * (lib.rs:333-353) is gpsb_resize to ceil(w/2) x ceil(h/2) plus gpsb_composite_rgba8 at w x h. */
typedef struct gpsb_session gpsb_session;
/* The renderer calls a session makes (gpsb_session_create binds them to a gpsb_renderer). */
typedef struct gpsb_session_backend {
    gpsb_status (*render_ensembles)(void* ctx, const gpsb_camera* cam, const gpsb_params* p, uint32_t first_seed,
                                    uint32_t count);
    gpsb_status (*render_sorted)(void* ctx, const gpsb_camera* cam, const gpsb_params* p, uint32_t as_ensembles);
    gpsb_status (*probe_demand)(void* ctx, const gpsb_camera* cam, const gpsb_params* p);
    gpsb_status (*request_stats)(void* ctx);
    gpsb_status (*latest_stats)(void* ctx, gpsb_stats* out);
    uint32_t (*stats_issued)(void* ctx);
    uint32_t (*accumulated)(void* ctx);
    uint32_t (*submitted)(void* ctx);
    gpsb_status (*reset_accum)(void* ctx);
    gpsb_status (*reset_stats)(void* ctx);
    uint32_t (*gaussian_count)(void* ctx);
} gpsb_session_backend;
typedef struct gpsb_session_state {
    uint32_t sorted_active, sorted_ok, moving_prefers_gps, lod_moving;
    uint32_t effective_per_frame, lod_n;
    float auto_density;
    uint32_t history_epoch, frames_since_reset, next_seed, ensemble_counter, slow_frames;
    uint64_t last_demand;
    double ema_ms;
} gpsb_session_state;
gpsb_status gpsb_session_create(gpsb_renderer* r, gpsb_session** out);
gpsb_status gpsb_session_create_with_backend(const gpsb_session_backend* backend, void* ctx, gpsb_session** out);
void gpsb_session_destroy(gpsb_session* s);
/* parameters (density clamped to 0.01..100, cap >= 1), ensembles per tick (1..4) and target */
gpsb_status gpsb_session_configure(gpsb_session* s, const gpsb_params* p, uint32_t per_frame, uint32_t target);
gpsb_status gpsb_session_set_lod(gpsb_session* s, int adaptive, double target_ms, uint32_t moving_cap);
gpsb_status gpsb_session_set_point_budget(gpsb_session* s, double millions);
/* mode 0 GPS particles, 1 depth-sorted, 2 Auto (GPS method only; PBVR always uses particles) */
gpsb_status gpsb_session_set_render_path(gpsb_session* s, uint32_t mode, double demand_threshold_millions);
/* camera of the next ticks (a different camera restarts the history); user_input marks motion */
gpsb_status gpsb_session_set_camera(gpsb_session* s, const gpsb_camera* cam, int user_input);
gpsb_status gpsb_session_reset(gpsb_session* s);
/* one tick at monotonic time now_ms; *presented = 1 when the accumulation changed */
gpsb_status gpsb_session_frame(gpsb_session* s, double now_ms, int* presented);
gpsb_status gpsb_session_read_state(const gpsb_session* s, gpsb_session_state* out);

/* ------------------------------------------------------------------- denoiser kernels
 * The learned denoiser of few-ensemble frames (the "denoised batch vs plain" comparison). The
 * reference has no denoiser, so none of these has a counterpart in it. All pointers are device
 * memory. The network's bf16 activations are chunk-planar, [B][C/8][H][W][8] (8-channel planes,
 * one pixel's 8 channels of a plane in 16 contiguous bytes), channel counts padded to multiples
 * of 8, a channel slice [off, off + n) being the planes off/8 ..; its fp32 buffers (gradients,
 * residual) are pixel-major [B][H][W][C]. An 8-channel tensor is the same in both layouts.
 * gpsb_dn_conv_fwd (the earlier engine) reads and writes pixel-major tensors. Weights are
 * (cout, kp) bf16 rows, k = (ky*3 + kx)*cin + ci, kp a multiple of 64 >= 9*cin. Work is enqueued on `stream` (a cudaStream_t, NULL = legacy default stream); the
 * return value is a cudaError_t code (0 = launched). `err` (a device word) receives a non-zero
 * bit when a bounded device-side wait gives up. */
/* y[p][ooff+n] = act(bias[n] + sum_k xcol[p][k] w[n][k]): 3x3 convolution, stride 1, zero padding
 * 1, on the tcgen05 tensor cores (implicit im2col through 16-byte copies); pixel-major x and out;
 * out is bf16, or fp32 when out_f32; relu != 0 applies ReLU. */
int gpsb_dn_conv_fwd(const void* x, int ldx, int xoff, int cin, int B, int H, int W, const void* w, int cout,
                     int kp, const float* bias, void* out, int ldo, int ooff, int out_f32, int relu,
                     void* stream, uint32_t* err);
/* The same convolution on chunk-planar activations with TMA-staged operands (persistent,
 * warp-specialised CTAs: one TMA box stages the input rows of an R-row x 128-pixel block as
 * 8-channel planes and the nine taps are shifted shared-memory descriptors over them; two
 * tensor-memory accumulators overlap the epilogue with the next block's MMAs). x: chunk-planar of
 * ldx channels; out: chunk-planar bf16 of ldo channels, or pixel-major fp32 (out_f32). Weights come
 * pre-arranged by gpsb_dn_conv3_weights into a buffer of gpsb_dn_conv3_weight_bytes(cout, cin)
 * bytes. x 16-byte aligned, ldx and xoff multiples of 8 (and ldo, ooff for bf16 out), cout <= 192;
 * a bounded device-side wait that gives up sets bit 32 of *err (err required). */
unsigned long long gpsb_dn_conv3_weight_bytes(int cout, int cin);
int gpsb_dn_conv3_weights(const void* w, int cout, int cin, int kp, void* wt, void* stream);
int gpsb_dn_conv3(const void* x, int ldx, int xoff, int cin, int B, int H, int W, const void* wt, int cout,
                  const float* bias, void* out, int ldo, int ooff, int out_f32, int relu, void* stream,
                  uint32_t* err);
/* dw[co][k] += sum_p dy[p][co] * xcol[p][k] (fp32, caller-zeroed): the weight gradient; dy and x
 * chunk-planar. */
int gpsb_dn_conv_dw(const void* dy, int ldy, const void* x, int ldx, int xoff, int cin, int B, int H, int W,
                    int cout, int kp, float* dw, void* stream, uint32_t* err);
/* wf[ci][(8 - t)*coutp + co] = w[co][t*cin + ci]: weights of the data gradient (a forward conv). */
int gpsb_dn_flip(const void* w, int cout, int cin, int kp, void* wf, int coutp, int kp2, void* stream);
/* out (chunk-planar bf16, ldo channels, B images of HW pixels) channel c = g[pix][goff+c] (fp32
 * pixel-major) * (y channel yoff+c > 0) (chunk-planar; y NULL: no mask) for c < C, zero above. */
int gpsb_dn_relu_bwd(const float* g, int ldg, int goff, const void* y, int ldy, int yoff, int B, int HW, int C,
                     void* out, int ldo, void* stream);
/* nearest 2x upsampling into a channel slice (chunk-planar), and its gradient (fp32 pixel-major,
 * sum over 2x2 blocks). */
int gpsb_dn_up2(const void* src, int lds, int B, int h, int w, int C, void* dst, int ldd, int doff, void* stream);
int gpsb_dn_up2_bwd(const float* g, int ldg, int goff, int B, int h, int w, int C, float* out, void* stream);
/* 2x2 average pooling of a channel slice (chunk-planar), and its gradient added into a channel
 * slice (fp32 pixel-major). */
int gpsb_dn_pool2(const void* src, int lds, int soff, int B, int h, int w, int C, void* dst, void* stream);
int gpsb_dn_pool2_bwd_add(const float* g, int B, int h, int w, int C, float* acc, int lda, int aoff,
                          void* stream);
/* db[c] += sum over the B x HW pixels of dz channel c (chunk-planar bf16 of ld channels, C <= 256). */
int gpsb_dn_bias_grad(const void* dz, int ld, int B, int HW, int C, float* db, void* stream);
/* L1 loss of base + r against target (M x 3 fp32): loss_sum += sum |d|; dr (M x 8 bf16) = scale*sign(d). */
int gpsb_dn_l1(const float* base, const float* r, const float* target, int M, float* loss_sum, void* dr,
               float scale, void* stream);
/* out = base + r (n floats). */
int gpsb_dn_residual(const float* base, const float* r, int n, float* out, void* stream);
/* Adam step t (>= 1) on n fp32 weights w with gradient g and moments m, v; wb (optional) gets bf16 w. */
int gpsb_dn_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                 int t, void* wb, void* stream);
/* dst[r][c] = bf16(c < cols ? src[r*lds + c] : 0) for c < ldd. */
int gpsb_dn_to_bf16(const float* src, int lds, int rows, int cols, void* dst, int ldd, void* stream);
/* Denoiser input of a frame: accum (P float4: rgb sum, count) and feature sums (P x 8 floats of
 * gpsb_set_feature_accum, or NULL) -> x (P x 8 bf16) and base (P x 3 fp32 mean colour). */
int gpsb_dn_pack(const void* accum, const float* feat, int P, void* x, float* base, void* stream);
/* Training crops: crops[3b..3b+2] = (image, y0, x0) windows of ch x cw from N stacked H x W frames
 * (B crops); a window outside the frames gives zeros and sets bit 16 of *err. */
int gpsb_dn_crop(const void* x, const float* base, const float* target, int N, int H, int W, const int* crops,
                 int B, int ch, int cw, void* xb, float* baseb, float* targetb, void* stream, uint32_t* err);

/* The denoised frame (no counterpart in the reference, which has no denoiser): the U-Net above,
 * sequenced on the host in C++ over these kernels, as one object with its weights and buffers.
 * Layers 0..10 are c1a c1b c2a c2b c3a c3b c4a c4b c5a c5b c6; gpsb_denoiser_layer_shape gives
 * each layer's padded and real input channels and its outputs. */
#define GPSB_DN_LAYERS 11
typedef struct gpsb_denoiser gpsb_denoiser;
gpsb_status gpsb_denoiser_create(int device, gpsb_denoiser** out);
void gpsb_denoiser_destroy(gpsb_denoiser* d);
const char* gpsb_denoiser_last_error(const gpsb_denoiser* d);
gpsb_status gpsb_denoiser_layer_shape(uint32_t layer, uint32_t* cin, uint32_t* cin_real, uint32_t* cout);
/* Host weights of one layer: w (cout x 9*cin floats, k = (ky*3 + kx)*cin + ci, cin the padded input
 * width) and b (cout floats): the "<name>.w" / "<name>.b" arrays of the committed weight file. */
gpsb_status gpsb_denoiser_set_layer(gpsb_denoiser* d, uint32_t layer, const float* w, const float* b);
/* The variance-check limit stored with the weights (mean per-pixel ensemble standard deviation). */
gpsb_status gpsb_denoiser_set_gate(gpsb_denoiser* d, float gate_limit);
/* The network on device tensors: x (width*height x 8 bf16 features of gpsb_dn_pack), base
 * (x 3 fp32 mean colour) -> pred_dev (x 3 fp32). Width and height multiples of 4. Synchronous. */
gpsb_status gpsb_denoiser_forward(gpsb_denoiser* d, const void* x_dev, const float* base_dev, uint32_t width,
                                  uint32_t height, float* pred_dev, void* cuda_stream);
/* How the network's layers run (gpsb_denoiser_forward, gpsb_render_denoised): 1 = captured in a
 * CUDA graph for the current frame size, later frames of that size replay it; 0 = no frame of the
 * current size yet (the next one launches the layers and captures them); -1 = a capture failed,
 * frames launch the layers directly. */
int gpsb_denoiser_graph_state(const gpsb_denoiser* d);
/* A denoised frame of renderer r (render_ensembles, crates/gps-render/src/gps.rs:861, followed by
 * the network): resets r's accumulation, renders `ensembles` ensembles (seeds first_seed..) with
 * per-pixel feature sums, packs the 8 input features and computes the variance check. When the
 * check is at most gate_limit (<= 0: the limit set with gpsb_denoiser_set_gate) the network's
 * prediction is returned (*used_denoiser = 1); otherwise the frame falls back to the plain
 * accumulation of fallback_ensembles ensembles (the next seeds are added to the same history;
 * *used_denoiser = 0). rgb_host: width*height*3 floats, linear RGB; *check: the check value.
 * Runs on r's stream and returns when the frame is in rgb_host. */
gpsb_status gpsb_render_denoised(gpsb_renderer* r, gpsb_denoiser* d, const gpsb_camera* cam, const gpsb_params* p,
                                 uint32_t first_seed, uint32_t ensembles, float gate_limit,
                                 uint32_t fallback_ensembles, float* rgb_host, int* used_denoiser, float* check);
/* Sum of channel c of a bf16 tensor (M x ld) added into *sum; rgb (P x 3) = accumulation / count. */
int gpsb_dn_channel_sum(const void* x, int ld, int c, int M, float* sum, void* stream);
int gpsb_dn_mean_rgb(const void* accum, int P, float* rgb, void* stream);

/* ------------------------------------------------------------------- PLY (gps-io) */
/* load_ply (crates/gps-io/src/lib.rs:260-338) + activation (lib.rs:84-96) +
 * GpuGaussian::from_activated (gps.rs:41-49), parsed on the host. Two calls: first with
 * outputs NULL to get n and the SH degree, then with buffers of n splats and
 * n*3*((d+1)^2-1) SH floats. */
gpsb_status gpsb_load_ply(const uint8_t* bytes, size_t len, size_t* n_out, uint32_t* sh_degree_out,
                          gpsb_gaussian* splats, float* sh_rest);
/* The same decode on the GPU for binary little-endian files (no counterpart in the reference,
 * which decodes on the host): the header is parsed on the host with gpsb_load_ply's rules and
 * messages, the vertex block is copied to the device once and decoded there one thread per
 * vertex into splats_dev (n x 64 bytes) and sh_rest_dev (n*3*((d+1)^2-1) floats), both device
 * memory, with the host loader's arithmetic; ready for gpsb_set_gaussians_sh_device. Two calls as
 * for gpsb_load_ply; ASCII files are refused (GPSB_ERR_PARSE). Synchronises `cuda_stream`. */
gpsb_status gpsb_load_ply_device(const uint8_t* bytes, size_t len, size_t* n_out, uint32_t* sh_degree_out,
                                 gpsb_gaussian* splats_dev, float* sh_rest_dev, void* cuda_stream);
/* Message of the last gpsb_load_ply failure on this thread (PlyError's Display, gps-io lib.rs:29-46). */
const char* gpsb_ply_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* GPSB200_H */
