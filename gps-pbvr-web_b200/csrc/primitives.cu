// Stand-alone primitives of the hot path, for the Phase-0 checks of the reference
// (crates/gps-render/src/lib.rs:99-275) and for HBM roofline measurements:
//   k_scan_u32_staged / k_scan_u32  single-pass decoupled-lookback exclusive scan of u32 counts
//                 (replaces the hierarchical scan_block/add_offsets of shaders/gps_scan.wgsl),
//                 64-bit total; the staged form for 16-byte aligned arrays, the other for the rest;
//   k_p0_sample   the synthetic two-pass atomicMin check of shaders/p0_sample.wgsl, with the
//                 packed 64-bit (key << 32 | colour) atomicMin that the particle kernel uses.
#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

namespace gpsb {

typedef unsigned long long ull;

#ifndef GPSB_SCAN_THREADS
#define GPSB_SCAN_THREADS 256
#endif
#ifndef GPSB_SCAN_ITEMS
#define GPSB_SCAN_ITEMS 24
#endif
#ifndef GPSB_SCAN_SLEEP
#define GPSB_SCAN_SLEEP 8
#endif
constexpr int kSThreads = GPSB_SCAN_THREADS;
constexpr int kSItems = GPSB_SCAN_ITEMS;  // a multiple of 4: 128-bit loads and stores
constexpr int kSTile = kSThreads * kSItems;
constexpr uint64_t kSAgg = 1ull << 62, kSPre = 2ull << 62, kSMask = (1ull << 62) - 1ull;

__device__ __forceinline__ uint64_t ld_rlx(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_rlx(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Decoupled lookback by warp 0 of a block (32 predecessors per round trip): publishes the tile's
// aggregate, sums predecessors' aggregates back to the nearest inclusive prefix, publishes the
// tile's inclusive prefix and returns the exclusive prefix (lane 0 holds it). Every wait is
// bounded; a predecessor that never publishes sets ERR_SCAN_LOOKBACK.
__device__ __forceinline__ uint64_t warp_lookback(uint64_t* lookback, uint32_t t, uint64_t agg, uint32_t* err) {
    const int lane = threadIdx.x & 31;
    uint64_t excl = 0;
    if (t == 0) {
        if (lane == 0) st_rlx(&lookback[0], kSPre | agg);
        return 0;
    }
    if (lane == 0) st_rlx(&lookback[t], kSAgg | agg);
    int32_t pred = (int32_t)t - 1;
    uint32_t spins = 0;
    bool failed = false;
    while (true) {
        int32_t j = pred - lane;
        uint64_t w = kSPre;  // before tile 0: an empty inclusive prefix
        if (j >= 0) {
            w = ld_rlx(&lookback[j]);
            while ((w >> 62) == 0ull) {
                if (++spins > (1u << 20)) { failed = true; break; }
                __nanosleep(GPSB_SCAN_SLEEP);
                w = ld_rlx(&lookback[j]);
            }
        }
        if (__any_sync(0xffffffffu, failed)) { failed = true; break; }
        uint32_t pre = __ballot_sync(0xffffffffu, (w >> 62) == 2ull);
        int first = pre ? __ffs(pre) - 1 : 32;
        uint64_t val = lane <= first ? (w & kSMask) : 0ull;
        for (int o = 16; o; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
        excl += val;
        if (first < 32) break;
        pred -= 32;
    }
    if (failed && lane == 0) atomicOr(err, ERR_SCAN_LOOKBACK);
    if (lane == 0) st_rlx(&lookback[t], kSPre | ((excl + agg) & kSMask));
    return excl;
}

// Each block scans kSTile consecutive counts (kSItems per thread, 128-bit loads), publishes its
// aggregate, looks back over its predecessors (warp 0, 32 at a time) and writes the exclusive
// prefix; the last tile writes the 64-bit total. Tile indices come from an atomic counter so
// every predecessor is running or done; waits are bounded and report through *err.
__global__ void __launch_bounds__(kSThreads) k_scan_u32(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                       uint32_t n, uint64_t* lookback, uint32_t* tile_counter,
                                                       uint32_t* err) {
    __shared__ uint32_t s_tile;
    __shared__ uint64_t s_w[kSThreads / 32];
    __shared__ uint64_t s_excl;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    const uint32_t base = t * kSTile + tid * kSItems;
    uint32_t v[kSItems];
    if (base + kSItems <= n && (((uintptr_t)(in + base)) & 15u) == 0) {
#pragma unroll
        for (int q = 0; q < kSItems; q += 4) {
            uint4 x = __ldcs(reinterpret_cast<const uint4*>(in + base + q));
            v[q] = x.x; v[q + 1] = x.y; v[q + 2] = x.z; v[q + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int q = 0; q < kSItems; ++q) v[q] = base + q < n ? in[base + q] : 0u;
    }
    uint64_t tsum = 0;
#pragma unroll
    for (int q = 0; q < kSItems; ++q) tsum += v[q];
    uint64_t incl = tsum;
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t a = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += a;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    uint64_t wpre = 0, agg = 0;
#pragma unroll
    for (int w = 0; w < kSThreads / 32; ++w) {
        if (w < warp) wpre += s_w[w];
        agg += s_w[w];
    }
    if (warp == 0) {
        uint64_t excl = warp_lookback(lookback, t, agg, err);
        if (lane == 0) s_excl = excl;
    }
    __syncthreads();
    uint64_t run = s_excl + wpre + (incl - tsum);
    uint32_t o[kSItems];
#pragma unroll
    for (int q = 0; q < kSItems; ++q) {
        o[q] = (uint32_t)run;
        run += v[q];
    }
    if (base + kSItems <= n && (((uintptr_t)(out + base)) & 15u) == 0) {
#pragma unroll
        for (int q = 0; q < kSItems; q += 4)
            __stcs(reinterpret_cast<uint4*>(out + base + q), make_uint4(o[q], o[q + 1], o[q + 2], o[q + 3]));
    } else {
#pragma unroll
        for (int q = 0; q < kSItems; ++q)
            if (base + q < n) out[base + q] = o[q];
    }
}

// Staged scan for 16-byte aligned arrays: tiles of 16384 counts (64 KB) so that one lookback
// round trip of warp 0 covers 2 MB of predecessors. Each thread copies 16-byte chunks of the tile
// (warp-consecutive, coalesced) into shared memory with cp.async, zero-filling past the end; the
// shared layout pads every 64-count thread segment by 16 bytes so that each thread then reads its
// own 64 consecutive counts without bank conflicts, sums them, and after the block scan and the
// lookback writes the exclusive prefixes back in place; the tile leaves through coalesced
// 16-byte stores. Three blocks (68 KB each) are resident per SM.
constexpr int kGThreads = 256;
constexpr int kGItems = 64;
constexpr int kGTile = kGThreads * kGItems;
constexpr int kGSeg = kGItems + 4;  // padded segment: an odd number of 16-byte chunks
constexpr size_t kGSmem = (size_t)kGThreads * kGSeg * 4;

__device__ __forceinline__ uint32_t staged_idx(uint32_t e) { return e + (e / kGItems) * 4u; }

__global__ void __launch_bounds__(kGThreads) k_scan_u32_staged(const uint32_t* __restrict__ in,
                                                              uint32_t* __restrict__ out, uint32_t n,
                                                              uint64_t* lookback, uint32_t* tile_counter,
                                                              uint32_t* err) {
    extern __shared__ __align__(128) uint32_t s_cnt[];  // kGThreads * kGSeg counts
    __shared__ uint32_t s_tile;
    __shared__ uint64_t s_w[kGThreads / 32];
    __shared__ uint64_t s_excl;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    const uint32_t tile0 = t * kGTile;
    const uint32_t cnt = n - tile0 < (uint32_t)kGTile ? n - tile0 : (uint32_t)kGTile;
#pragma unroll
    for (int k = 0; k < kGItems / 4; ++k) {
        const uint32_t e = (uint32_t)(k * kGThreads + tid) * 4u;
        const uint32_t bytes = e < cnt ? min(cnt - e, 4u) * 4u : 0u;  // < 16: the rest is zero-filled
        const uint32_t* src = bytes ? in + tile0 + e : in;
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(s_cnt + staged_idx(e));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    uint4* seg = reinterpret_cast<uint4*>(s_cnt + tid * kGSeg);
    uint64_t tsum = 0;
#pragma unroll
    for (int c = 0; c < kGItems / 4; ++c) {
        uint4 x = seg[c];
        tsum += (uint64_t)x.x + x.y + x.z + x.w;
    }
    uint64_t incl = tsum;
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t a = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += a;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    uint64_t wpre = 0, agg = 0;
#pragma unroll
    for (int w = 0; w < kGThreads / 32; ++w) {
        if (w < warp) wpre += s_w[w];
        agg += s_w[w];
    }
    if (warp == 0) {
        uint64_t excl = warp_lookback(lookback, t, agg, err);
        if (lane == 0) s_excl = excl;
    }
    __syncthreads();
    uint32_t run = (uint32_t)(s_excl + wpre + (incl - tsum));  // outputs are modulo 2^32
#pragma unroll
    for (int c = 0; c < kGItems / 4; ++c) {
        uint4 x = seg[c], o;
        o.x = run; run += x.x;
        o.y = run; run += x.y;
        o.z = run; run += x.z;
        o.w = run; run += x.w;
        seg[c] = o;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kGItems / 4; ++k) {
        const uint32_t e = (uint32_t)(k * kGThreads + tid) * 4u;
        const uint4 v = *reinterpret_cast<const uint4*>(s_cnt + staged_idx(e));
        if (e + 4u <= cnt) {
            __stcs(reinterpret_cast<uint4*>(out + tile0 + e), v);
        } else {
            if (e < cnt) out[tile0 + e] = v.x;
            if (e + 1u < cnt) out[tile0 + e + 1u] = v.y;
            if (e + 2u < cnt) out[tile0 + e + 2u] = v.z;
        }
    }
}

// The total is the inclusive prefix published by the last tile (status bits cleared).
__global__ void k_scan_total(uint64_t* total, const uint64_t* lookback, uint32_t tiles) {
    *total = lookback[tiles - 1] & kSMask;
}

uint32_t scan_tiles(uint32_t n) { return (n + kSTile - 1) / kSTile; }

void launch_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint64_t* lookback, uint32_t* counter,
                     uint64_t* total, uint32_t* err, cudaStream_t st) {
    uint32_t tiles = scan_tiles(n);
    cudaMemsetAsync(lookback, 0, (size_t)(tiles ? tiles : 1) * 8, st);
    cudaMemsetAsync(counter, 0, 4, st);
    if (n == 0) {
        if (total) cudaMemsetAsync(total, 0, 8, st);
        return;
    }
    if ((((uintptr_t)in) & 15u) == 0 && (((uintptr_t)out) & 15u) == 0) {
        // staged tiles are larger than kSTile, so the lookback words cleared above cover them
        const uint32_t gtiles = (n + kGTile - 1) / kGTile;
        cudaFuncSetAttribute(k_scan_u32_staged, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGSmem);
        k_scan_u32_staged<<<gtiles, kGThreads, kGSmem, st>>>(in, out, n, lookback, counter, err);
        if (total) k_scan_total<<<1, 1, 0, st>>>(total, lookback, gtiles);
        return;
    }
    k_scan_u32<<<tiles, kSThreads, 0, st>>>(in, out, n, lookback, counter, err);
    if (total) k_scan_total<<<1, 1, 0, st>>>(total, lookback, tiles);
}

// p0_sample.wgsl:26-39 gen_sample: pixel, ordered depth key (deliberately few values) and colour
__device__ __forceinline__ void p0_sample(uint32_t seed, uint32_t pixel_base, uint32_t pixels, uint32_t i, uint32_t* pix,
                                          uint32_t* key, uint32_t* rgb) {
    uint32_t h0 = gx::pcg(i ^ gx::pcg(seed));
    uint32_t h1 = gx::pcg(h0);
    uint32_t h2 = gx::pcg(h1);
    *pix = pixel_base + (h0 % pixels);
    uint32_t bits = 0x3F800000u | (h1 & 0x007FFFFFu);
    *key = (bits | 0x80000000u) & 0xFFFF0000u;
    *rgb = h2 & 0x00FFFFFFu;
}

__global__ void k_p0_sample(uint32_t seed, uint32_t pixel_base, uint32_t pixels, uint32_t samples, ull* packed) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= samples) return;
    uint32_t pix, key, rgb;
    p0_sample(seed, pixel_base, pixels, i, &pix, &key, &rgb);
    atomicMin(packed + pix, ((ull)key << 32) | rgb);
}

void launch_p0_sample(uint32_t seed, uint32_t pixel_base, uint32_t pixels, uint32_t samples, ull* packed, cudaStream_t st) {
    if (samples == 0) return;
    k_p0_sample<<<(samples + 255) / 256, 256, 0, st>>>(seed, pixel_base, pixels, samples, packed);
}

}  // namespace gpsb
