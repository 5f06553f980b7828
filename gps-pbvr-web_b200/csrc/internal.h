// Internal declarations shared by the kernels and the host renderer.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

#include "fmath.h"

namespace gpsb {

// Per-camera constants (the f32 part of FrameUniform, crates/gps-render/src/gps.rs:61-76,
// built by upload_frame gps.rs:812-856). The ensemble seed is first_seed + ensemble index and
// is passed separately so one FrameConst serves every ensemble of a camera.
struct FrameConst {
    float rot0[3], rot1[3], rot2[3];
    float pos[3];
    float low_pass;
    float fx, fy, cx, cy;
    uint32_t W, H, side, S, N;
    uint32_t cap;          // max(max_points_per_splat, 1)
    uint32_t sh_stride;    // SH coefficients per channel of the loaded scene
    uint32_t exact_radius;
    float density, near_z;
    float bg[3];
    uint32_t method, calibration, flags, sh_deg;
    float base_k, refl, object_depth;
    float jitter_sd;       // sqrt(max(low_pass, 0)), the low-pass jitter scale (gps_splat.wgsl:507)
    // footprint-subpixel Monte-Carlo mode of the CPU oracle (GPS only; fp_fixed <= 1 and
    // fp_kappa <= 0 = off): oracle.rs:203-235, lib.rs:412-433
    uint32_t fp_fixed, fp_max, fp_comp;
    float fp_kappa;
    uint32_t fast_mode;  // PBVR fast decisions: 0 off, 1 on, 2 validate (exact always, count disagreements)
};

enum : uint32_t { FLAG_RADIAL = 1u, FLAG_CENTRE = 2u, FLAG_JITTER = 4u };

// Count descriptor of one splat (8 bytes), written once per camera by the geometry kernel and
// read by the per-ensemble count+scan kernel.
//   mode 0: no particles;  1: Poisson(lambda) then the per-splat cap (GPS, PBVR);
//   2: exactly `fixed` particles, no cap (ScreenOccupancy dense);  3: Poisson(lambda), no cap
//   (ScreenOccupancy sparse). Bit 2 = under-covered (ViewConditioned).
enum : uint32_t { CD_NONE = 0u, CD_POISSON_CAP = 1u, CD_FIXED = 2u, CD_POISSON = 3u, CD_UNDERCOVERED = 4u };

// Particle record: 6 float4 per splat (the reference's proj layout, gps_splat.wgsl:627-628,
// 566-577, 605-610), plus hoisted per-splat constants in otherwise unused lanes:
//   GPS : r0 (mean.xy, depth, o)  r1 (l00, l10, l11, lut_a)  r2.x = bits(lut row i0), r2.y = Li2(o)
//   PBVR: r0 (mean.xy, depth, o)  r1.x keep, r1.y h(min(o, 1-1e-6))  r2 (pos, inv_xx)
//         r3 (inv_xy, inv_yy)  r4 (l00, l10, l11)  r5 (l20, l21, l22)
//   SO  : r0 (mean.xy, depth, o)  r1 (lo.xy, size.xy)  r2 (inv_xx, inv_xy, inv_yy, peak_tau)  r3.w sparse
constexpr int kRecF4 = 6;

// Statistics words (64-bit): gpsb_stats field order.
enum : int {
    ST_POINTS = 0, ST_TRUNCATED = 1, ST_DROPPED = 2, ST_VISIBLE = 3, ST_ORPHAN = 4, ST_CANDIDATES = 5,
    ST_UNDERCOVERED = 6, ST_SKIPPED = 7, ST_ENSEMBLES = 8, ST_PROBE = 9, ST_WRITES = 10, ST_ENTRIES = 11,
    ST_FAST_EXACT = 12, ST_FAST_MISMATCH = 13, ST_PARTICLES = 14, ST_WORDS = 16
};

// Device error word bits (bounded waits that gave up).
enum : uint32_t { ERR_SCAN_LOOKBACK = 1u, ERR_SORT_LOOKBACK = 2u, ERR_BAD_INDEX = 4u };

// Lookback word of the count scan: [63:62] status, [61:24] particle sum (saturating at 2^38),
// [23:0] number of splats with a non-zero count.
constexpr uint64_t kLbAggregate = 1ull << 62;
constexpr uint64_t kLbPrefix = 2ull << 62;
constexpr uint64_t kLbSumSat = (1ull << 38) - 1ull;

// Per-ensemble result of the count scan.
struct EnsTotal {
    uint64_t particles;   // saturating total (>= 2^32 means the u32 total overflowed)
    uint32_t nonzero;     // entries in the compact (splat id, offset) list
    uint32_t flags;       // bit0 overflow/skip, bit1 scan error
};

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kPartThreads = 256;
constexpr int kPartItems = 8;
constexpr int kPartTile = kPartThreads * kPartItems;

// ------------------------------------------------------------------ launchers (kernels.cu)
void launch_geometry(const FrameConst& fc, const float4* splats, const float* sh, const float* lut, float4* rec,
                     uint2* cdesc, float4* colour, cudaStream_t st);
void launch_count_scan(const FrameConst& fc, const uint2* cdesc, uint32_t first_seed, uint32_t E, uint64_t* lookback,
                       uint32_t* tile_counter, uint2* clist, EnsTotal* etot, unsigned long long* stats,
                       uint32_t* err, cudaStream_t st);
void launch_fast_bounds(uint32_t* out, cudaStream_t st);
void launch_particles(const FrameConst& fc, const float4* rec, const float* lut, const uint2* clist,
                      const EnsTotal* etot, uint32_t first_seed, uint32_t E, unsigned long long* sub,
                      uint32_t* unit_counter, unsigned long long* stats, int grid, int items, cudaStream_t st);
void launch_primitive(const FrameConst& fc, const float4* rec, const uint2* cdesc, const float* lut,
                      uint32_t first_seed, uint32_t E, unsigned long long* sub, EnsTotal* etot,
                      unsigned long long* stats, cudaStream_t st);
void launch_features(const FrameConst& fc, const unsigned long long* sub, const EnsTotal* etot, const float4* colour,
                     uint32_t E, float* feat, cudaStream_t st);
void launch_resolve(const FrameConst& fc, const unsigned long long* sub, const EnsTotal* etot, const float4* colour,
                    uint32_t E, float4* accum, unsigned long long* stats, cudaStream_t st);
void launch_add_stat(unsigned long long* stats, int word, unsigned long long v, cudaStream_t st);
void launch_debug_fmath(uint32_t which, const float* in, float* out, uint64_t n, cudaStream_t st);
void launch_debug_seeds(const uint2* list, uint32_t nonzero, uint64_t p0, uint32_t n, uint32_t seed, uint32_t* out,
                        cudaStream_t st);

// sorted path (sorted.cu)
struct SortedBuffers;
void launch_composite(const float4* accum, uint32_t W, uint32_t H, float exposure, uint32_t gamma_on, uint32_t out_w,
                      uint32_t out_h, uchar4* out, cudaStream_t st);

// stand-alone primitives (primitives.cu)
uint32_t scan_tiles(uint32_t n);
void launch_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint64_t* lookback, uint32_t* counter,
                     uint64_t* total, uint32_t* err, cudaStream_t st);
void launch_p0_sample(uint32_t seed, uint32_t pixel_base, uint32_t pixels, uint32_t samples, unsigned long long* packed,
                      cudaStream_t st);

int device_sm_count(int device);

}  // namespace gpsb
