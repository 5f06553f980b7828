// Direct 3x3 convolution (stride 1, zero padding 1) of chunk-planar bf16 activations on the tcgen05
// tensor cores, with every operand staged by TMA: the denoiser's forward layers and the data
// gradients of its backward pass (the same convolution with flipped weights).
//
// Activation layout in HBM ("chunk-planar"): a bf16 tensor of C channels (C a multiple of 8) over B
// images of H x W pixels is [B][C/8][H][W][8]: 8-channel chunk planes, each pixel's 8 channels of a
// chunk in 16 contiguous bytes, a row of a plane contiguous. A channel slice [off, off + n) (both
// multiples of 8) is a range of planes. fp32 outputs (the residual, the gradients) stay
// pixel-major [B][H][W][ld].
//
//   Y[b][y][x][n] = act(bias[n] + sum_{dy,dx,ci} X[b][y+dy][x+dx][ci] W[n][(dy+1)*3 + (dx+1)][ci])
//
// Work unit ("block"): R output rows x one 126-pixel row segment of one image, all N output
// channels. The K loop runs over groups of G input channels. One pipeline stage holds
//   * the R + 2 input rows y0-1 .. y0+R of the 128 pixels x0-1 .. x0+126 of the group's channels,
//     one plane per 8-channel chunk: [chunk][row][pixel][8 channels], 16 bytes per (row, pixel),
//     rows 2048 bytes apart. The chunk-planar tensor is viewed as 8-byte elements (2 per pixel) so
//     that the whole stage, 256 elements x (R + 2) rows x CH planes, is ONE TMA box: a TMA copy
//     costs about 80 clocks however small it is, and one copy per staged row (plus one for the
//     halo pixels a 128-pixel segment would need) bounded the narrow layers. Pixels, rows and
//     chunks outside the tensor read as zeros (TMA out-of-bounds fill), which is the padding;
//   * the group's weights in the canonical K-major layout of the MMA's B operand, one 1-D bulk copy
//     of a block that gpsb_dn_conv3_weights arranged once.
// In the canonical K-major layout without swizzle a core matrix is 8 rows x 16 bytes, i.e. eight
// consecutive pixels of one chunk plane; the MMA of output row r, tap (dy, dx) and chunk pair j
// reads A from plane 2j, row r + dy, starting at pixel dx (leading byte offset = the plane size,
// stride byte offset = 128 bytes): the nine taps are nine descriptors over the same staged rows,
// so each input byte crosses from L2 once per block instead of nine times. The MMA's M = 128 rows
// are output pixels x0 .. x0+127; the last two read past their staged row (into the next row, or
// for the last row of the last plane into the first bytes of the stage's weights) and are not
// stored, which is why a segment is 126 pixels.
//
// Cost of one MMA of M = 128, K = 16 (measured on B200, clocks): max(32 + N / 4, N / 2, ~40) on the
// tensor core (the 4 KB A tile and the N x 32-byte B tile read from shared memory at 128 bytes per
// clock, or the math), and about 54 clocks of issue for one thread. Narrow layers therefore
//   * stack the three vertical taps in one MMA when 3 N <= 256: staged row sr feeds output rows
//     sr - 2 .. sr, whose accumulators are consecutive column blocks, through B = the taps
//     dy = 2, 1, 0 stacked (weights arranged [dx][chunk][dy][n][8]), (R + 2) x 3 MMAs per chunk
//     pair instead of R x 9;
//   * for N <= 32, issue from two threads, each for its own half of the accumulator rows (the
//     stacked schedule clipped to those rows), so the order of every accumulation stays fixed.
//
// Roles (persistent CTAs, one per SM, 608 threads): warp 0 issues the TMA copies, lane 0 of warps 1
// (and 2) issues the MMAs (M = 128 pixels, N, K = 16) into one of two tensor-memory accumulators of
// R x N fp32 columns, warps 3-18 read the other accumulator back (tcgen05.ld, warp w reads lanes
// 32 (w % 4) .., four warps per lane quarter taking every fourth 32-column pair, two loads per
// wait) and apply bias (staged once per CTA in shared memory), ReLU and the bf16 / fp32 store, so
// the epilogue of block i overlaps the MMAs of block i + 1. Stages and accumulators hand over
// through mbarriers (TMA transaction counts, tcgen05.commit of each issuer, epilogue arrivals).
// Every wait is bounded: a wait that gives up sets bit CONV3_ERR_TIMEOUT in the caller's error word
// and raises an abort flag that ends every role; the CTA then waits (bounded) for its own TMA copies
// and MMAs before it frees its tensor memory and returns. No cluster, no multicast.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "pdl.cuh"
#include "umma.cuh"

namespace gpsb {
namespace c3 {

using bf16 = __nv_bfloat16;

constexpr int kSeg = 126;             // output pixels of a row segment (the MMA's M = 128, 2 unused)
constexpr int kStaged = 128;          // staged input pixels per row: x0 - 1 .. x0 + 126
constexpr int kRow = kStaged * 16;    // bytes of a staged row
constexpr int kThreads = 608;         // warp 0 TMA, warps 1-2 MMA, warps 3-18 epilogue
constexpr int kEpiWarps = 16;         // four per tensor-memory lane quarter
constexpr int kEpiWarp0 = 3;          // first epilogue warp
constexpr uint32_t kAccCols = 256;    // tensor-memory columns of one accumulator (two are allocated)
constexpr uint32_t kSpin = 1u << 24;  // polls of a bounded wait
constexpr uint32_t CONV3_ERR_TIMEOUT = 32u;

__host__ __device__ constexpr int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Per output-channel width N and chunk planes per stage CHS: R rows per block (R x N <= 256
// accumulator columns), G = 8 CHS channels per stage, S stages, the byte layout of a stage, and
// whether the three vertical taps share one MMA (STACK: 3 N <= 256, see the MMA issuer).
template <int N, int CHS>
struct Cfg {
    static constexpr int R = N <= 32 ? 8 : N <= 64 ? 4 : N <= 128 ? 2 : 1;
    static constexpr int CH = CHS;                                       // chunk planes per stage
    static constexpr int G = 8 * CH;
    static constexpr bool STACK = 3 * N <= 256;
    // MMA-issuing threads: one thread issues at most one M = 128 MMA per ~54 clocks, while the
    // tensor core finishes one of N <= 32 in ~40 (its 4 KB A read), so for N <= 32 two threads
    // issue, each for its own half of the accumulator rows
    static constexpr int ISSUERS = (STACK && R == 8) ? 2 : 1;
    static constexpr int PLANE = (R + 2) * kRow;                         // bytes of one chunk plane
    static constexpr int IN = CH * PLANE;                                // staged input rows of a stage
    static constexpr int WB = 9 * CH * N * 16;                           // weight bytes of one group
    static constexpr int STAGE = round_up(IN + WB, 1024);                // a stage with its group's weights
    static constexpr int STAGE_IN = round_up(IN, 1024);                  // a stage of input rows only
    static constexpr int S = N >= 192 ? 3 : 2;
    static constexpr uint32_t TX = (uint32_t)(IN + WB);                  // bytes landing per stage
    static constexpr size_t SMEM = (size_t)S * STAGE + 1024;             // + alignment slack
    // the layout with every group's weights resident (one copy per CTA): S input stages + weights
    static constexpr size_t smem_resident(int groups) { return (size_t)S * STAGE_IN + (size_t)groups * WB + 1024; }
    static_assert(R * N <= (int)kAccCols, "accumulator columns");
    static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N of one MMA");
    static_assert(SMEM <= 232448, "shared memory per CTA");
    static_assert(CH % 2 == 0, "an MMA reads two chunk planes (K = 16)");
};

// chunk planes per stage of the instance serving N outputs and cin inputs
__host__ __device__ constexpr int chs_of(int N, int cin) { return (N >= 192 || cin <= 16) ? 2 : 4; }

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, K-major, no swizzle (sm_100 descriptor version 1)
__device__ __forceinline__ uint64_t desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ bool bar_test(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase of parity `parity`; gives up when the limit passes or another role
// raised the abort flag.
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity, volatile int* abort) {
    for (uint32_t i = 0; i < kSpin; ++i) {
        if (bar_test(b, parity)) return true;
        if ((i & 255u) == 255u && *abort) return false;
    }
    return false;
}
__device__ __forceinline__ void bar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(b)) : "memory");
}
__device__ __forceinline__ void bar_expect(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
// one 4-D TMA tile load into shared memory, completion counted on the mbarrier
__device__ __forceinline__ void tma_load4(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                          uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(saddr(bar))
        : "memory");
}
// one contiguous bulk copy global -> shared (16-byte aligned, size a multiple of 16)
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(saddr(bar))
                 : "memory");
}

struct Params {
    const bf16* wt;       // arranged weights: [group][tap][chunk][n][8]
    const float* bias;    // [cout] or null
    void* out;            // bf16: chunk-planar [B][ldo/8][H][W][8]; fp32: [B][H][W][ldo]; channels from ooff
    int ldo, ooff, out_f32, relu;
    int B, H, W, cout, groups;
    int segs, rowblocks, blocks;
    int resident;  // every group's weights stay in shared memory after one copy per CTA
    uint32_t* err;
};

// Bias, ReLU and the store of output channels c .. c + 15 of pixel (b, y, x): v the 16 accumulator
// columns, bias the 16 staged bias values (16-byte aligned).
__device__ __forceinline__ void store16(const Params& p, float* v, const float* bias, int b, int y, int x, int c) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 bq = reinterpret_cast<const float4*>(bias)[q];
        v[4 * q] += bq.x;
        v[4 * q + 1] += bq.y;
        v[4 * q + 2] += bq.z;
        v[4 * q + 3] += bq.w;
    }
    if (p.relu) {
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = fmaxf(v[k], 0.0f);
    }
    const size_t pix = ((size_t)b * p.H + y) * p.W + x;
    if (p.out_f32) {
        float* o = reinterpret_cast<float*>(p.out) + pix * p.ldo + p.ooff + c;
        if (c + 16 <= p.cout && ((p.ldo | p.ooff) & 3) == 0) {
            float4* dst = reinterpret_cast<float4*>(o);
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        } else {
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if (c + k < p.cout) o[k] = v[k];
        }
        return;
    }
    // chunk-planar: output channels ooff + c .. + 15 are two 16-byte pixel slots of planes
    // (ooff + c) / 8 and + 1 (a warp stores 32 consecutive pixels of a plane)
    bf16* o = reinterpret_cast<bf16*>(p.out);
    const size_t plane = (size_t)p.H * p.W, img = (size_t)y * p.W + x, base_b = (size_t)b * (p.ldo / 8);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int n0 = c + 8 * h;
        if (n0 >= p.cout) break;
        const size_t at = ((base_b + (size_t)((p.ooff + n0) >> 3)) * plane + img) * 8;
        if (n0 + 8 <= p.cout) {
            uint32_t w[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                __nv_bfloat162 hh = __floats2bfloat162_rn(v[8 * h + 2 * q], v[8 * h + 2 * q + 1]);
                w[q] = *reinterpret_cast<uint32_t*>(&hh);
            }
            *reinterpret_cast<uint4*>(o + at) = make_uint4(w[0], w[1], w[2], w[3]);
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (n0 + k < p.cout) o[at + k] = __float2bfloat16_rn(v[8 * h + k]);
        }
    }
}

template <int N, int CHS>
__global__ void __launch_bounds__(kThreads, 1) k_conv3(const __grid_constant__ CUtensorMap xmap,
                                                     const Params p) {
    using C = Cfg<N, CHS>;
    extern __shared__ __align__(1024) uint8_t s_raw[];
    __shared__ __align__(8) uint64_t s_full[C::S], s_empty[C::S], s_acc_full[2], s_acc_empty[2], s_drain[2], s_wbar;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    __shared__ __align__(16) float s_bias[N];  // bias of the N accumulator columns (0 past cout)
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(s_raw) + 1023) & ~(uintptr_t)1023);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // stage s at base + s * stride; resident weights (group g at wres + g WB) after the S stages
    const size_t stride = p.resident ? (size_t)C::STAGE_IN : (size_t)C::STAGE;
    uint8_t* const wres = base + (size_t)C::S * C::STAGE_IN;

    // Launched with programmatic stream serialisation, this prologue (tensor memory, barriers, the
    // tensor-map prefetch) overlaps the end of the previous kernel; nothing in global memory is read
    // before the grid-dependency wait (the previous kernel may have written the input, the weights
    // or the bias), and every write comes after it.
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&s_tmem)),
                     "r"(2u * kAccCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        if (lane == 0) asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&xmap)) : "memory");
    }
    if (tid == 32) {
        for (int s = 0; s < C::S; ++s) {
            bar_init(&s_full[s], 1);
            bar_init(&s_empty[s], C::ISSUERS);
        }
        for (int a = 0; a < 2; ++a) {
            bar_init(&s_acc_full[a], C::ISSUERS);
            bar_init(&s_acc_empty[a], kEpiWarps);
        }
        bar_init(&s_drain[0], 1);
        bar_init(&s_drain[1], 1);
        bar_init(&s_wbar, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    grid_dependency_wait();
    launch_dependents();
    for (int n = tid; n < N; n += kThreads) s_bias[n] = (p.bias && n < p.cout) ? p.bias[n] : 0.0f;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    auto fail = [&]() {
        if (!s_abort) {
            s_abort = 1;
            atomicOr(p.err, CONV3_ERR_TIMEOUT);
        }
    };
    // block -> (image, first output row, first output pixel)
    auto decode = [&](int blk, int& b, int& y0, int& x0) {
        const int seg = blk % p.segs, rb = (blk / p.segs) % p.rowblocks;
        b = blk / (p.segs * p.rowblocks);
        y0 = rb * C::R;
        x0 = seg * kSeg;
    };

    if (warp == 0) {
        // ------------------------------------------------------------------ TMA producer
        // lane 0: wait for a free stage, arm its barrier, issue the stage's one input box and the
        // group's weights
        if (lane == 0) {
            if (p.resident) {
                bar_expect(&s_wbar, (uint32_t)(p.groups * C::WB));
                for (int g = 0; g < p.groups; ++g)
                    bulk_load(saddr(wres) + (uint32_t)(g * C::WB), p.wt + (size_t)g * (C::WB / 2), (uint32_t)C::WB, &s_wbar);
            }
            uint32_t armed = 0;  // stages armed at least once (for the abort drain)
            int stage = 0;
            uint32_t phase = 0;
            bool stop = false;
            for (int blk = blockIdx.x; blk < p.blocks && !stop; blk += gridDim.x) {
                int b, y0, x0;
                decode(blk, b, y0, x0);
                for (int g = 0; g < p.groups; ++g) {
                    if (s_abort || !bar_wait(&s_empty[stage], phase ^ 1u, &s_abort)) {
                        fail();
                        stop = true;
                        break;
                    }
                    bar_expect(&s_full[stage], p.resident ? (uint32_t)C::IN : C::TX);
                    const uint32_t st = saddr(base + (size_t)stage * stride);
                    tma_load4(st, &xmap, 2 * (x0 - 1), y0 - 1, g * C::CH, b, &s_full[stage]);
                    if (!p.resident)
                        bulk_load(st + C::IN, p.wt + (size_t)g * (C::WB / 2), (uint32_t)C::WB, &s_full[stage]);
                    armed |= 1u << stage;
                    if (++stage == C::S) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            if (s_abort) {
                // let this CTA's copies land before the CTA can exit: every stage's last armed phase
                // (and the resident weights' barrier) completes by its transaction count alone
                if (p.resident) {
                    for (uint32_t i = 0; i < kSpin && !bar_test(&s_wbar, 0); ++i) {
                    }
                }
                int st2 = stage;
                uint32_t ph2 = phase;
                for (int k = 0; k < C::S; ++k) {
                    if (--st2 < 0) {
                        st2 = C::S - 1;
                        ph2 ^= 1u;
                    }
                    if (armed & (1u << st2)) {
                        for (uint32_t i = 0; i < kSpin && !bar_test(&s_full[st2], ph2); ++i) {
                        }
                    }
                }
            }
        }
        __syncwarp();
    } else if (warp < kEpiWarp0) {
        // ------------------------------------------------------------------ MMA issuers
        // lane 0 of warp 1 + h issues the MMAs of accumulator rows [rlo, rhi] of every block
        const int h = warp - 1;
        constexpr int kRows = C::R / C::ISSUERS;
        const int rlo = h * kRows, rhi = rlo + kRows - 1;
        if (lane == 0 && h < C::ISSUERS) {
            constexpr uint32_t idesc = umma::idesc_bf16(N);
            int stage = 0, a = 0;
            uint32_t phase = 0, aphase = 0;
            bool issued = false;
            if (p.resident) {
                if (bar_wait(&s_wbar, 0, &s_abort)) asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                else fail();
            }
            for (int blk = blockIdx.x; blk < p.blocks && !s_abort; blk += gridDim.x) {
                if (!bar_wait(&s_acc_empty[a], aphase ^ 1u, &s_abort)) {
                    fail();
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)a * kAccCols;
                bool ok = true;
                for (int g = 0; g < p.groups; ++g) {
                    if (!bar_wait(&s_full[stage], phase, &s_abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t st = saddr(base + (size_t)stage * stride);
                    const uint32_t wg = p.resident ? saddr(wres) + (uint32_t)(g * C::WB) : st + C::IN;
                    // one descriptor per operand and stage; every MMA adds a compile-time byte
                    // offset / 16 to its 14-bit start-address field (shared addresses stay below
                    // 256 KB, so the field never carries into the offsets above it)
                    if constexpr (C::STACK) {
                        // Staged row sr (image row y0 - 1 + sr) feeds output rows sr - 2, sr - 1, sr
                        // through the vertical taps dy = 2, 1, 0. The group's B operand of (dx, chunk)
                        // holds the three taps' N x 8 blocks stacked in that order, so one MMA of
                        // width (hi - lo + 1) N writes the accumulators of output rows lo .. hi, which
                        // lie in consecutive N-column blocks. Output row sr is first written by staged
                        // row sr (tap dy = 0) at dx = 0, first chunk pair, group 0: that block is split
                        // off and written without accumulation.
                        const uint64_t a0 = desc(st, C::PLANE, 128), b0 = desc(wg, 3 * N * 16, 128);
                        constexpr uint32_t id1 = umma::idesc_bf16(N), id2 = umma::idesc_bf16(2 * N),
                                           id3 = umma::idesc_bf16(3 * N);
#pragma unroll 1
                        for (int sr = rlo; sr < rhi + 3; ++sr) {
                            const int lo = sr - 2 > rlo ? sr - 2 : rlo, hi = sr < rhi ? sr : rhi;
                            const int rows = hi - lo + 1;
                            const uint32_t idn = rows == 3 ? id3 : rows == 2 ? id2 : id1;
                            const uint32_t dlo = acc + (uint32_t)(lo * N);
                            const int boff = (lo - sr + 2) * N;  // stacked row of output row lo's tap
                            const uint64_t ar = a0 + (uint64_t)(sr * (kRow / 16));
                            const bool fresh = g == 0 && hi == sr;
#pragma unroll
                            for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
                                for (int j = 0; j < C::CH / 2; ++j) {
                                    const uint64_t ad = ar + (uint64_t)(2 * j * (C::PLANE / 16) + dx);
                                    const uint64_t bt = b0 + (uint64_t)((dx * C::CH + 2 * j) * 3 * N);
                                    if (dx == 0 && j == 0 && fresh) {
                                        umma::mma_bf16(acc + (uint32_t)(sr * N), ad, bt + 2 * N, id1, false);
                                        if (lo < sr) umma::mma_bf16(dlo, ad, bt + boff, rows == 3 ? id2 : id1, true);
                                    } else {
                                        umma::mma_bf16(dlo, ad, bt + boff, idn, true);
                                    }
                                }
                            }
                        }
                    } else {
                        const uint64_t a0 = desc(st, C::PLANE, 128), b0 = desc(wg, N * 16, 128);
#pragma unroll 1
                        for (int r = rlo; r <= rhi; ++r) {
                            const uint64_t ar = a0 + (uint64_t)(r * (kRow / 16));
                            const uint32_t d = acc + (uint32_t)(r * N);
#pragma unroll
                            for (int t = 0; t < 9; ++t) {
                                constexpr int kRow16 = kRow / 16;
                                const int dy = t / 3, dx = t % 3;  // input row r + dy, pixel offset dx (staged from -1)
#pragma unroll
                                for (int j = 0; j < C::CH / 2; ++j) {
                                    const uint64_t ad = ar + (uint64_t)(2 * j * (C::PLANE / 16) + dy * kRow16 + dx);
                                    const uint64_t bd = b0 + (uint64_t)((t * C::CH + 2 * j) * N);
                                    umma::mma_bf16(d, ad, bd, idesc, g > 0 || t > 0 || j > 0);
                                }
                            }
                        }
                    }
                    umma::mma_commit(&s_empty[stage]);  // frees the stage when these MMAs complete
                    issued = true;
                    if (++stage == C::S) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) {
                    fail();
                    break;
                }
                umma::mma_commit(&s_acc_full[a]);
                if (++a == 2) {
                    a = 0;
                    aphase ^= 1u;
                }
            }
            // every MMA this CTA issued has completed before its tensor memory can be freed
            if (issued) {
                umma::mma_commit(&s_drain[h]);
                for (uint32_t i = 0; i < kSpin && !bar_test(&s_drain[h], 0); ++i) {
                }
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------------ epilogue (warps 3-18)
        // the accumulator of a block is R x N columns = R N / 32 pairs of 16-column units (unit u:
        // output row u / (N / 16), channels 16 (u % (N / 16)) ..); warp w reads tensor-memory lanes
        // 32 (w % 4) .. (its 32 pixels), so four warps share each lane quarter and take every fourth
        // pair (two loads, one wait)
        constexpr int kPairs = C::R * N / 32;
        constexpr int kMine = (kPairs + 3) / 4;  // pairs per warp, at most
        static_assert(C::R * N % 32 == 0, "whole pairs of 16-column units");
        const int quad = warp & 3, part = (warp - kEpiWarp0) >> 2;
        const int px = quad * 32 + lane;
        int a = 0;
        uint32_t aphase = 0;
        for (int blk = blockIdx.x; blk < p.blocks && !s_abort; blk += gridDim.x) {
            int b, y0, x0;
            decode(blk, b, y0, x0);
            if (!bar_wait(&s_acc_full[a], aphase, &s_abort)) {
                fail();
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int x = x0 + px;
            const uint32_t lane_base = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)a * kAccCols;
#pragma unroll
            for (int i = 0; i < kMine; ++i) {
                const int pr = part + 4 * i;  // warp-uniform
                if (pr >= kPairs) break;
                float v[32];
                umma::tmem_ld16_issue(lane_base + (uint32_t)(pr * 32), v);
                umma::tmem_ld16_issue(lane_base + (uint32_t)(pr * 32 + 16), v + 16);
                umma::tmem_ld_wait(v);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int u = 2 * pr + h, y = y0 + u / (N / 16), c = (u % (N / 16)) * 16;
                    if (px < kSeg && x < p.W && y < p.H) store16(p, v + 16 * h, s_bias + c, b, y, x, c);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) bar_arrive(&s_acc_empty[a]);
            if (++a == 2) {
                a = 0;
                aphase ^= 1u;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2u * kAccCols) : "memory");
}

// Weights of one layer in the order the kernel streams them (zero past cin or cout; w: [cout][kp]
// bf16, K index k = tap * cin + ci, tap = 3 dy + dx):
//   wt[g][t][c][n][e]      = w[n][t * cin + g G + 8 c + e]                     (N >= 96)
//   wt[g][dx][c][s][n][e]  = w[n][(3 (2 - s) + dx) * cin + g G + 8 c + e]      (stacked, N <= 64)
__global__ void k_conv3_arrange(const bf16* w, int cout, int cin, int kp, int N, int G, int groups, int stack,
                                bf16* wt) {
    const int CH = G / 8;
    const long total = (long)groups * 9 * CH * N * 8;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        long q = i;
        const int e = (int)(q % 8);
        q /= 8;
        const int n = (int)(q % N);
        q /= N;
        int t, c, g;
        if (stack) {
            const int s3 = (int)(q % 3);
            q /= 3;
            c = (int)(q % CH);
            q /= CH;
            const int dx = (int)(q % 3);
            g = (int)(q / 3);
            t = 3 * (2 - s3) + dx;
        } else {
            c = (int)(q % CH);
            q /= CH;
            t = (int)(q % 9);
            g = (int)(q / 9);
        }
        const int ci = g * G + c * 8 + e;
        bf16 v = __float2bfloat16_rn(0.0f);
        if (n < cout && ci < cin) v = w[(size_t)n * kp + t * cin + ci];
        wt[i] = v;
    }
}

// N of the kernel instance serving `cout` output channels
static int n_of(int cout) {
    if (cout <= 16) return 16;
    if (cout <= 32) return 32;
    if (cout <= 64) return 64;
    if (cout <= 96) return 96;
    if (cout <= 128) return 128;
    return 192;
}
static int g_of(int N, int cin) { return 8 * chs_of(N, cin); }

static PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    });
    return fn;
}

template <int N, int CHS>
static cudaError_t launch(const bf16* x, int ldx, int xoff, int cin, const Params& prm, cudaStream_t st) {
    using Cf = Cfg<N, CHS>;
    auto enc = encoder();
    if (!enc) return cudaErrorNotSupported;
    // 4-D view of the chunk-planar activations as 8-byte elements: (2 W, H, chunk, B), the chunks of
    // channels [xoff, xoff + cin) of a tensor of ldx channels; the box of one stage: 256 elements
    // (128 pixels) x (R + 2) rows x CH chunk planes
    CUtensorMap map;
    const cuuint64_t plane = (cuuint64_t)prm.W * prm.H * 16;  // bytes of one chunk plane
    const cuuint64_t dims[4] = {(cuuint64_t)prm.W * 2, (cuuint64_t)prm.H, (cuuint64_t)((cin + 7) / 8), (cuuint64_t)prm.B};
    const cuuint64_t strides[3] = {(cuuint64_t)prm.W * 16, plane, plane * (cuuint64_t)(ldx / 8)};
    const cuuint32_t box[4] = {2 * kStaged, (cuuint32_t)Cf::R + 2, (cuuint32_t)Cf::CH, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    void* gaddr = (void*)(x + (size_t)(xoff / 8) * prm.W * prm.H * 8);
    const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, gaddr, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    Params q = prm;
    q.segs = (prm.W + kSeg - 1) / kSeg;
    q.rowblocks = (prm.H + Cf::R - 1) / Cf::R;
    q.blocks = q.segs * q.rowblocks * prm.B;
    q.groups = (cin + Cf::G - 1) / Cf::G;
    int dev = 0, sms = 148, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, k_conv3<N, CHS>);
    if (e != cudaSuccess) return e;
    // the largest dynamic size this instance may use (set once to the maximum, so every launch of
    // it, captured in a graph or not, stays within the attribute)
    const size_t dyn_max = (size_t)optin - fa.sharedSizeBytes;
    if (Cf::SMEM > dyn_max) return cudaErrorInvalidConfiguration;
    e = cudaFuncSetAttribute(k_conv3<N, CHS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_max);
    if (e != cudaSuccess) return e;
    const size_t smem_res = Cf::smem_resident(q.groups);
    q.resident = smem_res <= dyn_max ? 1 : 0;
    const size_t smem = q.resident ? smem_res : Cf::SMEM;
    const int grid = q.blocks < sms ? q.blocks : sms;
    if (grid <= 0) return cudaSuccess;
    return launch_pdl(k_conv3<N, CHS>, dim3(grid), dim3(kThreads), smem, st, map, q);
}

}  // namespace c3
}  // namespace gpsb

using namespace gpsb;
using namespace gpsb::c3;

extern "C" {

// Bytes of the arranged weights of a layer with cout outputs and cin inputs (see k_conv3_arrange).
unsigned long long gpsb_dn_conv3_weight_bytes(int cout, int cin) {
    if (cout < 1 || cout > 192 || cin < 1) return 0;
    const int N = n_of(cout), G = g_of(N, cin);
    return (unsigned long long)((cin + G - 1) / G) * 9ull * (G / 8) * N * 16ull;
}

// Arranges w ([cout][kp] bf16, k = tap * cin + ci) into wt (gpsb_dn_conv3_weight_bytes bytes).
int gpsb_dn_conv3_weights(const void* w, int cout, int cin, int kp, void* wt, void* stream) {
    if (cout < 1 || cout > 192 || cin < 1 || kp < 9 * cin || !w || !wt) return (int)cudaErrorInvalidValue;
    const int N = n_of(cout), G = g_of(N, cin), groups = (cin + G - 1) / G;
    const long total = (long)groups * 9 * (G / 8) * N * 8;
    const int blocks = (int)((total + 255) / 256 < 1184 ? (total + 255) / 256 : 1184);
    k_conv3_arrange<<<blocks, 256, 0, (cudaStream_t)stream>>>((const bf16*)w, cout, cin, kp, N, G, groups,
                                                              3 * N <= 256 ? 1 : 0, (bf16*)wt);
    return (int)cudaGetLastError();
}

// 3x3 convolution, stride 1, zero padding 1: chunk-planar bf16 input x of ldx channels (B, H, W),
// channels [xoff, xoff + cin), arranged weights wt, output channels [ooff, ooff + cout) of a tensor
// of ldo channels: bf16 chunk-planar (ooff a multiple of 8), or fp32 pixel-major (out_f32);
// optional bias and ReLU. ldx, xoff multiples of 8, x 16-byte aligned, cout <= 192. Enqueues on
// `stream`; a device-side wait that gives up sets bit 32 of *err.
int gpsb_dn_conv3(const void* x, int ldx, int xoff, int cin, int B, int H, int W, const void* wt, int cout,
                  const float* bias, void* out, int ldo, int ooff, int out_f32, int relu, void* stream, uint32_t* err) {
    if (!x || !wt || !out || !err || ldx % 8 || xoff % 8 || cin < 1 || xoff + cin > ldx || cout < 1 || cout > 192 ||
        B < 1 || H < 1 || W < 1 || ooff < 0 || ooff + cout > ldo || (reinterpret_cast<uintptr_t>(x) & 15u) ||
        (!out_f32 && (ldo % 8 || ooff % 8)))
        return (int)cudaErrorInvalidValue;
    Params prm{};
    prm.wt = (const bf16*)wt;
    prm.bias = bias;
    prm.out = out;
    prm.ldo = ldo;
    prm.ooff = ooff;
    prm.out_f32 = out_f32;
    prm.relu = relu;
    prm.B = B;
    prm.H = H;
    prm.W = W;
    prm.cout = cout;
    prm.err = err;
    const bf16* xb = (const bf16*)x;
    cudaStream_t st = (cudaStream_t)stream;
    const bool narrow = chs_of(32, cin) == 2;  // cin <= 16: two chunk planes per stage
    switch (n_of(cout)) {
        case 16: return (int)(narrow ? launch<16, 2>(xb, ldx, xoff, cin, prm, st) : launch<16, 4>(xb, ldx, xoff, cin, prm, st));
        case 32: return (int)(narrow ? launch<32, 2>(xb, ldx, xoff, cin, prm, st) : launch<32, 4>(xb, ldx, xoff, cin, prm, st));
        case 64: return (int)(narrow ? launch<64, 2>(xb, ldx, xoff, cin, prm, st) : launch<64, 4>(xb, ldx, xoff, cin, prm, st));
        case 96: return (int)(narrow ? launch<96, 2>(xb, ldx, xoff, cin, prm, st) : launch<96, 4>(xb, ldx, xoff, cin, prm, st));
        case 128: return (int)(narrow ? launch<128, 2>(xb, ldx, xoff, cin, prm, st) : launch<128, 4>(xb, ldx, xoff, cin, prm, st));
        default: return (int)launch<192, 2>(xb, ldx, xoff, cin, prm, st);
    }
}

}  // extern "C"
