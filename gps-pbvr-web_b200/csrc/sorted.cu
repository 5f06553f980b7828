// Depth-sorted alpha path and the radix sort, for sm_100a.
//
//   k_sp_project    sp_project (gps_splat.wgsl:737-777): 24-bit far-to-near key, quad record,
//                   GPS demand probe, plus the screen-tile rectangle of the splat.
//   radix_sort_pairs  stable LSD onesweep sort (replaces gps_sort.wgsl): one histogram pass for
//                   all digits, then one kernel per digit that ranks keys within each warp by
//                   peer groups (each lane ORs its bit into its digit's word of a per-warp row in
//                   shared memory and reads the word back), resolves tile offsets by a decoupled
//                   lookback per digit and scatters. Digit width 4, 6 or 8 bits.
//   tile binning    (tile id, sorted rank) entries, stably sorted by tile, give every screen tile its
//                   splats in depth order.
//   k_blend         one block per tile, front-to-back f32 blending with early termination
//                   (replaces the rgba16f back-to-front raster of gps_sorted_draw.wgsl:15-38 and the
//                   blend state of sorted.rs:125-138), written to accum = (rgb, 1) like sp_resolve.
//   k_composite     gps_composite.wgsl:41-55 into a headless RGBA8 buffer.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <mutex>

#include "../../include/gpsb200.h"
#include "devmath.cuh"
#include "sorted.h"

namespace gpsb {

typedef unsigned long long ull;

__device__ __forceinline__ uint32_t ld_relaxed32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed32(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ============================================================================ radix sort
constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
// Keys per thread and resident blocks per SM of a onesweep pass, per digit width: 8-bit digits
// take 25 keys per thread (6400 per tile, 62.5 KB of staging, 3 blocks per SM), whose longer
// digit runs write out in fuller sectors (2^26 pairs: 15 keys 2.24 TB/s, 21 2.31, 23 2.41, 25
// 2.47); 4- and 6-bit digits 15 (3840, 37.5 KB, 4 blocks per SM), where larger tiles gained nothing.
#ifndef GPSB_SORT_IPT8
#define GPSB_SORT_IPT8 25
#endif
#ifndef GPSB_SORT_IPT
#define GPSB_SORT_IPT 15
#endif
template <int BITS>
struct RsShape {
    static constexpr int ipt = BITS >= 8 ? GPSB_SORT_IPT8 : GPSB_SORT_IPT;
    static constexpr int tile = kRsThreads * ipt;
    static constexpr size_t stage = (size_t)tile * 10;  // dynamic shared memory of one block
    static constexpr int min_blocks = stage + 8 * 1024 > 56 * 1024 ? 3 : 4;
    static_assert(tile % 4 == 0 && tile <= 65536, "tile staging layout");
};
constexpr int kMaxPasses = 8;
#ifndef GPSB_SORT_LOOKAHEAD
#define GPSB_SORT_LOOKAHEAD 8
#endif
constexpr int kRsLook = GPSB_SORT_LOOKAHEAD;  // predecessor tiles read per lookback round trip
#ifndef GPSB_SORT_BALLOT_PEERS
// 0 match.any, 1 ballots, 2 alternating per key, 3 shared-memory OR (2^26 pairs, 8-bit digits:
// ballots 1.421 ms, shared OR 1.368, with the bulk value copy 1.330; A/B on one B200)
#define GPSB_SORT_BALLOT_PEERS 3
#endif
constexpr uint32_t kStAgg = 1u << 30, kStPre = 2u << 30, kStMask = (1u << 30) - 1u;
#ifndef GPSB_SORT_BULK_VALUES
#define GPSB_SORT_BULK_VALUES 1  // 1: a full tile's values arrive by one cp.async.bulk (mbarrier), 0: 16-byte cp.async
#endif

template <int BITS>
__global__ void __launch_bounds__(256) k_radix_hist(const uint32_t* __restrict__ keys, uint32_t n, int passes,
                                                    uint32_t* hist) {
    constexpr int BINS = 1 << BITS;
    __shared__ uint32_t s[kMaxPasses * BINS];
    for (int k = threadIdx.x; k < passes * BINS; k += blockDim.x) s[k] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t k = __ldg(&keys[i]);
        for (int p = 0; p < passes; ++p) atomicAdd(&s[p * BINS + ((k >> (p * BITS)) & (BINS - 1))], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < passes * BINS; k += blockDim.x)
        if (s[k]) atomicAdd(&hist[k], s[k]);
}

// exclusive scan of every pass's histogram, in place (one block)
template <int BITS>
__global__ void k_radix_hist_scan(uint32_t* hist, int passes) {
    constexpr int BINS = 1 << BITS;
    int p = threadIdx.x;
    if (p >= passes) return;
    uint32_t acc = 0;
    for (int d = 0; d < BINS; ++d) {
        uint32_t c = hist[p * BINS + d];
        hist[p * BINS + d] = acc;
        acc += c;
    }
}

template <int BITS>
__global__ void __launch_bounds__(kRsThreads, RsShape<BITS>::min_blocks) k_onesweep(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                         uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                         uint32_t n, int shift, const uint32_t* __restrict__ gstart,
                                                         uint32_t* lookback, uint32_t* tile_counter, uint32_t* err) {
    constexpr int BINS = 1 << BITS;
    constexpr int kRsIpt = RsShape<BITS>::ipt, kRsTile = RsShape<BITS>::tile;
    __shared__ uint32_t s_wcnt[kRsWarps][BINS];  // per-warp digit counts, then exclusive prefix over warps
    __shared__ uint32_t s_dstart[BINS];          // tile-local exclusive prefix over digits
    __shared__ uint32_t s_gbase[BINS];           // global position of the digit's first key of this tile, minus s_dstart
    // dynamic shared memory (RsShape::stage bytes): keys in digit order, the tile's values in input order
    // (16-byte aligned for cp.async), the tile-local input index of each ordered key
    extern __shared__ __align__(16) uint32_t s_stage[];
    uint32_t* s_key = s_stage;
    uint32_t* s_vin = s_stage + kRsTile;
    uint16_t* s_src = reinterpret_cast<uint16_t*>(s_stage + 2 * kRsTile);
    __shared__ uint32_t s_wsum[kRsWarps];
    __shared__ uint32_t s_tile;
    __shared__ __align__(8) uint64_t s_vbar;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s_tile = atomicAdd(tile_counter, 1u);
        if (GPSB_SORT_BULK_VALUES) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(&s_vbar))
                         : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    for (int k = tid; k < kRsWarps * BINS; k += kRsThreads) (&s_wcnt[0][0])[k] = 0;
    __syncthreads();
    const uint32_t t = s_tile;
    const uint32_t tile0 = t * kRsTile;
    const uint32_t tile_n = n - tile0 < (uint32_t)kRsTile ? n - tile0 : (uint32_t)kRsTile;
    const uint32_t base = tile0 + warp * 32 * kRsIpt;
    // the tile's values travel to shared memory asynchronously while the keys are ranked
    const bool vasync = (((uintptr_t)vin) & 15u) == 0;
    const bool vbulk = GPSB_SORT_BULK_VALUES && vasync && tile_n == (uint32_t)kRsTile;
    if (vbulk) {
        if (tid == 0) {
            const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&s_vbar);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kRsTile * 4u)
                         : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             (uint32_t)__cvta_generic_to_shared(s_vin)),
                         "l"(vin + tile0), "r"(kRsTile * 4u), "r"(bar)
                         : "memory");
        }
    } else if (!vasync) {
        for (uint32_t e = tid; e < tile_n; e += kRsThreads) s_vin[e] = vin[tile0 + e];
    } else {
        for (uint32_t c = tid; c < (uint32_t)kRsTile / 4u; c += kRsThreads) {
            const uint32_t e = c * 4u;
            const uint32_t bytes = e < tile_n ? min(tile_n - e, 4u) * 4u : 0u;
            const uint32_t* src = bytes ? vin + tile0 + e : vin;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                             (uint32_t)__cvta_generic_to_shared(s_vin + e)),
                         "l"(src), "r"(bytes)
                         : "memory");
        }
    }
    uint32_t key[kRsIpt], rank[kRsIpt];
    const uint32_t lt = lanemask_lt();
    uint32_t* wc = s_wcnt[warp];
    // peer masks through shared memory (variant 3): each warp's row of BINS words lives in the key
    // staging area, which the ranking does not use yet (it is written after the block barrier that
    // ends the ranking); rows start at zero and every group's lowest lane clears its digit's word
    uint32_t* wm = s_key + warp * BINS;
    if (GPSB_SORT_BALLOT_PEERS == 3) {
        for (int k = lane; k < BINS; k += 32) wm[k] = 0u;
        __syncwarp();
    }
    // rank every key within its warp's sub-tile in input order (stable): the lanes holding one digit
    // find each other (peers: one ballot per digit bit, or match.any), every lane reads its digit's
    // running count of the warp, and the lowest lane of each group adds the group's size (the
    // groups hold distinct digits, so the warp's counter row needs no atomics)
    auto rank_key = [&](int q, uint32_t d, uint32_t live) {
        uint32_t peers;
        if (GPSB_SORT_BALLOT_PEERS == 3) {
            if ((live >> lane) & 1u) atomicOr(&wm[d], 1u << lane);
            __syncwarp();
            peers = wm[d] & live;
        } else if (GPSB_SORT_BALLOT_PEERS == 1 || (GPSB_SORT_BALLOT_PEERS == 2 && (q & 1))) {
            peers = live;
#pragma unroll
            for (int b = 0; b < BITS; ++b) {
                const bool bs = (d >> b) & 1u;
                const uint32_t m = __ballot_sync(0xffffffffu, bs);
                peers &= bs ? m : ~m;
            }
        } else {
            peers = __match_any_sync(0xffffffffu, d) & live;
        }
        const uint32_t below = __popc(peers & lt);
        const uint32_t old = wc[d];
        __syncwarp();
        if (below == 0u && ((live >> lane) & 1u)) {
            wc[d] = old + (uint32_t)__popc(peers);
            if (GPSB_SORT_BALLOT_PEERS == 3) wm[d] = 0u;
        }
        __syncwarp();  // orders this key's count update before the next key's reads
        rank[q] = old + below;
    };
    if (tile_n == (uint32_t)kRsTile) {
        const uint32_t* kp = kin + base + lane;  // the keys of this lane, 32 apart
#pragma unroll
        for (int q = 0; q < kRsIpt; ++q) {
            key[q] = __ldg(kp + q * 32);
            rank_key(q, (key[q] >> shift) & (BINS - 1), 0xffffffffu);
        }
    } else {
#pragma unroll
        for (int q = 0; q < kRsIpt; ++q) {
            const uint32_t idx = base + q * 32 + lane;
            const bool valid = idx < n;
            key[q] = valid ? __ldg(&kin[idx]) : 0u;
            rank_key(q, valid ? ((key[q] >> shift) & (BINS - 1)) : 0u, __ballot_sync(0xffffffffu, valid));
        }
    }
    __syncthreads();
    // per digit: exclusive prefix over warps and the tile count; publish the tile's aggregate early
    uint32_t* lb = lookback + (size_t)t * BINS;
    uint32_t cnt = 0;
    if (tid < BINS) {
#pragma unroll
        for (int w = 0; w < kRsWarps; ++w) {
            uint32_t c = s_wcnt[w][tid];
            s_wcnt[w][tid] = cnt;
            cnt += c;
        }
        st_relaxed32(&lb[tid], (t == 0 ? kStPre : kStAgg) | cnt);
    }
    // exclusive scan of the digit counts over the tile (BINS <= 256 = one value per thread)
    uint32_t incl = tid < BINS ? cnt : 0u;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t a = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += a;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += s_wsum[w];
    if (tid < BINS) s_dstart[tid] = wbase + incl - cnt;
    if (vbulk) {
        if (tid == 0) {  // the bulk copy has landed (bounded wait); the barrier below shares it
            const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&s_vbar);
            uint32_t ok = 0;
            for (uint32_t i = 0; i < (1u << 24) && !ok; ++i)
                asm volatile(
                    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}"
                    : "=r"(ok)
                    : "r"(bar)
                    : "memory");
            if (!ok) atomicOr(err, ERR_SORT_LOOKBACK);
        }
    } else if (vasync) {
        asm volatile("cp.async.wait_all;" ::: "memory");  // own copies done; the barrier shares them
    }
    __syncthreads();
    // scatter into shared memory in digit order (stable); values follow through their input index
#pragma unroll
    for (int q = 0; q < kRsIpt; ++q) {
        uint32_t idx = base + q * 32 + lane;
        if (idx < n) {
            uint32_t d = (key[q] >> shift) & (BINS - 1);
            uint32_t pos = s_dstart[d] + s_wcnt[warp][d] + rank[q];
            s_key[pos] = key[q];
            s_src[pos] = (uint16_t)(idx - tile0);
        }
    }
    // lookback per digit, kRsLook predecessors per round trip; an unpublished word is polled again
    if (tid < BINS) {
        uint32_t excl = 0;
        if (t > 0) {
            int32_t pred = (int32_t)t - 1;
            uint32_t spins = 0;
            bool failed = false;
            while (true) {
                uint32_t w[kRsLook];
#pragma unroll
                for (int u = 0; u < kRsLook; ++u)
                    w[u] = pred - u >= 0 ? ld_relaxed32(&lookback[(size_t)(pred - u) * BINS + tid]) : kStPre;
                int used = 0;
                bool done = false;
#pragma unroll
                for (int u = 0; u < kRsLook; ++u) {
                    if (done || used < u || (w[u] >> 30) == 0u) continue;
                    excl += w[u] & kStMask;
                    used = u + 1;
                    done = (w[u] >> 30) == 2u;
                }
                if (done) break;
                pred -= used;
                if (used < kRsLook) {
                    if (++spins > (1u << 22)) { failed = true; break; }
                    __nanosleep(32);
                }
            }
            if (failed) atomicOr(err, ERR_SORT_LOOKBACK);
            st_relaxed32(&lb[tid], kStPre | ((excl + cnt) & kStMask));
        }
        s_gbase[tid] = gstart[tid] + excl - s_dstart[tid];
    }
    __syncthreads();
    // coalesced write-out: consecutive threads write consecutive keys of each digit run
    // (a position past n would mean corrupt histograms: it is skipped and reported once per thread)
    bool bad = false;
    auto write_one = [&](uint32_t i) {
        const uint32_t k = s_key[i];
        const uint32_t pos = s_gbase[(k >> shift) & (BINS - 1)] + i;
        const bool ok = pos < n;
        bad |= !ok;
        if (ok) {
            kout[pos] = k;
            vout[pos] = s_vin[s_src[i]];
        }
    };
    if (tile_n == (uint32_t)kRsTile) {
#pragma unroll
        for (int q = 0; q < kRsIpt; ++q) write_one((uint32_t)(q * kRsThreads + tid));
    } else {
        for (uint32_t i = tid; i < tile_n; i += kRsThreads) write_one(i);
    }
    if (bad) atomicOr(err, ERR_BAD_INDEX);
}

void radix_release(RadixScratch& s) {
    if (s.hist) cudaFree(s.hist);
    if (s.lookback) cudaFree(s.lookback);
    if (s.counters) cudaFree(s.counters);
    s = RadixScratch();
}

// One onesweep pass; the staging lives in dynamic shared memory (above 48 KB for large tiles).
template <int BITS>
static void onesweep_launch(uint32_t tiles, const uint32_t* ik, const uint32_t* iv, uint32_t* ok, uint32_t* ov,
                            uint32_t n, int shift, const uint32_t* gstart, uint32_t* lookback, uint32_t* counter,
                            uint32_t* err, cudaStream_t st) {
    // set on every launch: the attributes belong to the current device's context
    cudaFuncSetAttribute(k_onesweep<BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RsShape<BITS>::stage);
    cudaFuncSetAttribute(k_onesweep<BITS>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    k_onesweep<BITS><<<tiles, kRsThreads, RsShape<BITS>::stage, st>>>(ik, iv, ok, ov, n, shift, gstart, lookback, counter, err);
}

template <int BITS>
static cudaError_t radix_impl(RadixScratch& s, uint32_t* ka, uint32_t* va, uint32_t* kb, uint32_t* vb, uint32_t n,
                              int key_bits, uint32_t* err, cudaStream_t st) {
    constexpr int BINS = 1 << BITS;
    int passes = std::max(1, (key_bits + BITS - 1) / BITS);
    if (passes > kMaxPasses) return cudaErrorInvalidValue;
    const uint32_t tiles = (n + RsShape<BITS>::tile - 1) / RsShape<BITS>::tile;
    size_t hb = (size_t)passes * BINS * 4, lbb = (size_t)passes * std::max(tiles, 1u) * BINS * 4;
    cudaError_t e;
    if (hb > s.hist_bytes) {
        if (s.hist) cudaFree(s.hist);
        s.hist = nullptr;
        if ((e = cudaMalloc(&s.hist, hb)) != cudaSuccess) return e;
        s.hist_bytes = hb;
    }
    if (lbb > s.lookback_bytes) {
        if (s.lookback) cudaFree(s.lookback);
        s.lookback = nullptr;
        if ((e = cudaMalloc(&s.lookback, lbb)) != cudaSuccess) return e;
        s.lookback_bytes = lbb;
    }
    if (!s.counters && (e = cudaMalloc(&s.counters, kMaxPasses * 4)) != cudaSuccess) return e;
    uint32_t* hist = (uint32_t*)s.hist;
    cudaMemsetAsync(hist, 0, hb, st);
    cudaMemsetAsync(s.lookback, 0, lbb, st);
    cudaMemsetAsync(s.counters, 0, kMaxPasses * 4, st);
    if (n == 0) return cudaGetLastError();
    k_radix_hist<BITS><<<std::min<uint32_t>((n + 4095) / 4096, 1184u), 256, 0, st>>>(ka, n, passes, hist);
    k_radix_hist_scan<BITS><<<1, 32, 0, st>>>(hist, passes);
    // ping-pong so that the last pass writes (kb, vb)
    uint32_t *ik = ka, *iv = va, *ok = kb, *ov = vb;
    if (passes % 2 == 0) { ok = ka; ov = va; ik = kb; iv = vb; }
    if (passes % 2 == 0) {
        // first pass reads the input from (ka, va): copy it to (kb, vb) so the parity works out
        cudaMemcpyAsync(kb, ka, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vb, va, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
    }
    for (int p = 0; p < passes; ++p) {
        onesweep_launch<BITS>(tiles, ik, iv, ok, ov, n, p * BITS, hist + p * BINS,
                              (uint32_t*)s.lookback + (size_t)p * tiles * BINS, (uint32_t*)s.counters + p, err, st);
        std::swap(ik, ok);
        std::swap(iv, ov);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------- no-allocation sort
// Callers that may not allocate device memory (a host application that owns the whole GPU memory
// budget through its own pool, or a real-time frame loop where a cudaMalloc would stall or is
// forbidden) use gpsb_sort_pairs_noalloc. Its scratch (digit histograms, tile counters and the
// lookback words) is this file-scope array, sized for kNoAllocMaxN pairs with up to 32-bit keys
// (4 passes of 8-bit digits): about 1.35 MB that every GPU which loads the library keeps until the
// process exits.
constexpr uint32_t kNoAllocMaxN = 1u << 21;
constexpr uint32_t kNoAllocTiles = (kNoAllocMaxN + RsShape<8>::tile - 1) / RsShape<8>::tile;
constexpr uint32_t kNoAllocPasses = 4;
constexpr size_t kNoAllocHistWords = kNoAllocPasses * 256;
constexpr size_t kNoAllocCounterWords = 16;  // per-pass tile counters (padded)
constexpr size_t kNoAllocWords = kNoAllocHistWords + kNoAllocCounterWords + (size_t)kNoAllocPasses * kNoAllocTiles * 256;
static __device__ __align__(256) uint32_t g_noalloc_sort_scratch[kNoAllocWords];

cudaError_t radix_sort_pairs(RadixScratch& s, uint32_t* ka, uint32_t* va, uint32_t* kb, uint32_t* vb, uint32_t n,
                             int key_bits, int digit_bits, uint32_t* err, cudaStream_t st) {
    if (digit_bits == 4) return radix_impl<4>(s, ka, va, kb, vb, n, key_bits, err, st);
    if (digit_bits == 6) return radix_impl<6>(s, ka, va, kb, vb, n, key_bits, err, st);
    return radix_impl<8>(s, ka, va, kb, vb, n, key_bits, err, st);
}

// Device address of g_noalloc_sort_scratch on the current device. In host code the array's name is
// only a host-side stand-in, so the address comes from cudaGetSymbolAddress with the device
// current. It is looked up again on every call whose stream is not capturing (so a device reset,
// which reloads the module, never leaves a stale address behind) and kept per device ordinal for
// calls made while `st` is being captured into a graph, which must follow one uncaptured call.
static void* noalloc_scratch_address(cudaStream_t st, cudaError_t* err, bool* capture_without_setup) {
    static std::mutex mu;
    static void* addr[256] = {};
    *capture_without_setup = false;
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess) return nullptr;
    if (dev < 0 || dev >= 256) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    *err = cudaStreamIsCapturing(st, &cs);
    if (*err != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (cs == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        *err = cudaGetSymbolAddress(&p, g_noalloc_sort_scratch);
        if (*err != cudaSuccess) return nullptr;
        addr[dev] = p;
    } else if (!addr[dev]) {
        *capture_without_setup = true;
    }
    return addr[dev];
}

// ============================================================================ u32 exclusive scan
constexpr int kScT = 256, kScI = 8, kScTile = kScT * kScI;

__global__ void __launch_bounds__(kScT) k_scan_reduce(const uint32_t* __restrict__ in, uint32_t n, uint32_t* sums) {
    __shared__ uint32_t s[kScT / 32];
    uint32_t base = blockIdx.x * kScTile, v = 0;
    for (int q = 0; q < kScI; ++q) {
        uint32_t i = base + q * kScT + threadIdx.x;
        if (i < n) v += in[i];
    }
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kScT / 32; ++w) t += s[w];
        sums[blockIdx.x] = t;
    }
}
// single block: exclusive scan of the block sums (nb <= 1024 * 16), total into *total
__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t* sums, uint32_t nb, uint32_t* total) {
    __shared__ uint32_t s[1024];
    const int per = (nb + 1023) / 1024;
    uint32_t loc = 0;
    for (int q = 0; q < per; ++q) {
        uint32_t i = threadIdx.x * per + q;
        if (i < nb) loc += sums[i];
    }
    s[threadIdx.x] = loc;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        uint32_t v = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
        __syncthreads();
        s[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = s[threadIdx.x] - loc;
    for (int q = 0; q < per; ++q) {
        uint32_t i = threadIdx.x * per + q;
        if (i < nb) {
            uint32_t c = sums[i];
            sums[i] = run;
            run += c;
        }
    }
    if (threadIdx.x == 1023) *total = s[1023];
}
__global__ void __launch_bounds__(kScT) k_scan_apply(uint32_t* data, uint32_t n, const uint32_t* sums) {
    __shared__ uint32_t s[kScT];
    uint32_t base = blockIdx.x * kScTile + threadIdx.x * kScI;
    uint32_t v[kScI], t = 0;
    for (int q = 0; q < kScI; ++q) {
        v[q] = base + q < n ? data[base + q] : 0u;
        t += v[q];
    }
    s[threadIdx.x] = t;
    __syncthreads();
    for (int o = 1; o < kScT; o <<= 1) {
        uint32_t a = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
        __syncthreads();
        s[threadIdx.x] += a;
        __syncthreads();
    }
    uint32_t run = sums[blockIdx.x] + s[threadIdx.x] - t;
    for (int q = 0; q < kScI; ++q) {
        if (base + q < n) data[base + q] = run;
        run += v[q];
    }
}

// ============================================================================ sorted path
struct TileGeom {
    uint32_t tw, th, tiles_x, tiles_y;
};

// sp_project (gps_splat.wgsl:737-777) + tile rectangle
__global__ void __launch_bounds__(128) k_sp_project(FrameConst f, TileGeom tg, const float4* __restrict__ splats,
                                                     const float* __restrict__ sh, uint32_t* keys, uint32_t* vals,
                                                     float4* rec, uint2* rect, ull* stats, int full) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    ull demand = 0;
    if (i < f.N) {
        if (full) {
            keys[i] = 0xFFFFFFu;
            vals[i] = i;
            rect[i] = make_uint2(0xFFFFFFFFu, 0u);
        }
        float4 g0 = __ldg(&splats[4 * (size_t)i]), g1 = __ldg(&splats[4 * (size_t)i + 1]);
        float4 g2 = __ldg(&splats[4 * (size_t)i + 2]), g3 = __ldg(&splats[4 * (size_t)i + 3]);
        Proj pr = project(f, g0, g1, g2);
        float o = clamp_(g0.w, F_(0.0), F_(1.0));
        bool vis = pr.ok && o > F_(0.0);
        if (vis) {
            float ex = gxc::kOffscreenSigma * sqrt_(pr.a), ey = gxc::kOffscreenSigma * sqrt_(pr.c);
            vis = !(pr.mx + ex < F_(0.0) || pr.mx - ex >= (float)f.W || pr.my + ey < F_(0.0) || pr.my - ey >= (float)f.H);
        }
        if (vis) {
            float det = pr.a * pr.c - pr.b * pr.b;
            float en = f.density * (float)f.S * F_(2.0) * gxc::kPi * sqrt_(det) * dilog(o);
            if (en > F_(0.0)) demand = f2u(fmin_(en, F_(4.0e9)));
        }
        if (full && vis && !(o < gxc::kSpMinAlpha)) {
            float K = sqrt_(F_(2.0) * gx::log(div_(o, gxc::kSpMinAlpha)));
            float ex = K * sqrt_(pr.a), ey = K * sqrt_(pr.c);
            if (!(pr.mx + ex < F_(0.0) || pr.mx - ex >= (float)f.W || pr.my + ey < F_(0.0) || pr.my - ey >= (float)f.H)) {
                float tr2 = F_(0.5) * (pr.a + pr.c);
                float disc = sqrt_(fmax_(tr2 * tr2 - (pr.a * pr.c - pr.b * pr.b), F_(0.0)));
                float l1 = tr2 + disc;
                float l2 = fmax_(tr2 - disc, F_(1e-12));
                float v1x = F_(1.0), v1y = F_(0.0);
                if (fabsf(pr.b) > F_(1e-12)) {
                    float ux = l1 - pr.c, uy = pr.b;
                    float len = sqrt_(ux * ux + uy * uy);
                    v1x = div_(ux, len);
                    v1y = div_(uy, len);
                } else if (pr.a < pr.c) {
                    v1x = F_(0.0);
                    v1y = F_(1.0);
                }
                float v2x = -v1y, v2y = v1x;
                float s1 = sqrt_(l1), s2 = sqrt_(l2);
                rec[3 * (size_t)i] = make_float4(pr.mx, pr.my, o, K);
                rec[3 * (size_t)i + 1] = make_float4(div_(v1x, s1), div_(v1y, s1), div_(v2x, s2), div_(v2y, s2));
                rec[3 * (size_t)i + 2] = splat_colour(f, sh, i, g0, g3);
                keys[i] = 0xFFFFFEu - (f2b(pr.depth) >> 8u);
                // pixel-centre bounding box of the ellipse r2 <= K^2, padded, in tiles
                float bx = K * sqrtf(l1 * v1x * v1x + l2 * v2x * v2x) * 1.001f + 1.0f;
                float by = K * sqrtf(l1 * v1y * v1y + l2 * v2y * v2y) * 1.001f + 1.0f;
                float x0f = floorf(pr.mx - bx - 0.5f), x1f = ceilf(pr.mx + bx - 0.5f);
                float y0f = floorf(pr.my - by - 0.5f), y1f = ceilf(pr.my + by - 0.5f);
                if (x1f >= 0.0f && y1f >= 0.0f && x0f <= (float)(f.W - 1) && y0f <= (float)(f.H - 1)) {
                    uint32_t x0 = (uint32_t)fmaxf(x0f, 0.0f), y0 = (uint32_t)fmaxf(y0f, 0.0f);
                    uint32_t x1 = (uint32_t)fminf(x1f, (float)(f.W - 1)), y1 = (uint32_t)fminf(y1f, (float)(f.H - 1));
                    rect[i] = make_uint2((x0 / tg.tw) | ((y0 / tg.th) << 16), (x1 / tg.tw) | ((y1 / tg.th) << 16));
                }
            }
        }
    }
    for (int o = 16; o; o >>= 1) demand += __shfl_xor_sync(0xffffffffu, demand, o);
    if ((threadIdx.x & 31) == 0 && demand) atomicAdd(&stats[ST_PROBE], demand);
}

__device__ __forceinline__ uint32_t rect_tiles(uint2 r) {
    if (r.x == 0xFFFFFFFFu) return 0u;
    uint32_t w = (r.y & 0xFFFFu) - (r.x & 0xFFFFu) + 1u, h = (r.y >> 16) - (r.x >> 16) + 1u;
    return w * h;
}

__global__ void k_gather_counts(const uint32_t* __restrict__ keys_sorted, const uint32_t* __restrict__ vals_sorted,
                                const uint2* __restrict__ rect, uint32_t n, uint32_t* cnt) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    cnt[j] = keys_sorted[j] == 0xFFFFFFu ? 0u : rect_tiles(rect[vals_sorted[j]]);
}

__global__ void k_emit_entries(const uint32_t* __restrict__ keys_sorted, const uint32_t* __restrict__ vals_sorted,
                               const uint2* __restrict__ rect, const uint32_t* __restrict__ offs, uint32_t n,
                               uint32_t tiles_x, uint32_t* ekey, uint32_t* eval) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || keys_sorted[j] == 0xFFFFFFu) return;
    uint2 r = rect[vals_sorted[j]];
    if (r.x == 0xFFFFFFFFu) return;
    uint32_t o = offs[j];
    for (uint32_t ty = r.x >> 16; ty <= (r.y >> 16); ++ty)
        for (uint32_t tx = r.x & 0xFFFFu; tx <= (r.y & 0xFFFFu); ++tx) {
            ekey[o] = ty * tiles_x + tx;
            eval[o] = j;
            ++o;
        }
}

__global__ void k_tile_ranges(const uint32_t* __restrict__ ekey, uint32_t m, uint2* ranges) {
    uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= m) return;
    uint32_t t = ekey[o];
    if (o == 0 || ekey[o - 1] != t) ranges[t].x = o;
    if (o == m - 1 || ekey[o + 1] != t) ranges[t].y = o + 1;
}

// One block per screen tile: pixels blend their tile's splats nearest first.
template <int TW, int TH>
__global__ void __launch_bounds__(TW* TH) k_blend(uint32_t W, uint32_t H, uint32_t tiles_x, const uint2* __restrict__ ranges,
                                                 const uint32_t* __restrict__ erank, const uint32_t* __restrict__ vals_sorted,
                                                 const float4* __restrict__ rec, float bg0, float bg1, float bg2,
                                                 float4* accum) {
    constexpr int NT = TW * TH;
    __shared__ float4 s_a[NT], s_b[NT], s_c[NT];
    const uint32_t tile = blockIdx.x;
    const uint32_t px = (tile % tiles_x) * TW + threadIdx.x % TW, py = (tile / tiles_x) * TH + threadIdx.x / TW;
    const bool inside = px < W && py < H;
    const float pcx = (float)px + F_(0.5), pcy = (float)py + F_(0.5);
    const uint2 range = ranges[tile];
    float T = F_(1.0), cr = F_(0.0), cg = F_(0.0), cb = F_(0.0);
    bool done = !inside;
    for (int end = (int)range.y; end > (int)range.x; end -= NT) {
        int cnt = min(NT, end - (int)range.x);
        __syncthreads();
        if ((int)threadIdx.x < cnt) {
            uint32_t id = __ldg(&vals_sorted[__ldg(&erank[end - 1 - threadIdx.x])]);
            s_a[threadIdx.x] = __ldg(&rec[3 * (size_t)id]);
            s_b[threadIdx.x] = __ldg(&rec[3 * (size_t)id + 1]);
            s_c[threadIdx.x] = __ldg(&rec[3 * (size_t)id + 2]);
        }
        __syncthreads();
        if (!done) {
            for (int q = 0; q < cnt; ++q) {
                float4 a = s_a[q], b = s_b[q];
                float dx = pcx - a.x, dy = pcy - a.y;
                float u = dx * b.x + dy * b.y;
                float v = dx * b.z + dy * b.w;
                float r2 = u * u + v * v;
                if (r2 > a.w * a.w) continue;
                float alpha = fmin_(a.z * gx::exp(-F_(0.5) * r2), F_(0.99));
                if (alpha < gxc::kSpMinAlpha) continue;
                float4 c = s_c[q];
                float wgt = T * alpha;
                cr = cr + wgt * c.x;
                cg = cg + wgt * c.y;
                cb = cb + wgt * c.z;
                T = T * (F_(1.0) - alpha);
                if (T < F_(1e-4)) {
                    done = true;
                    break;
                }
            }
        }
        if (__syncthreads_count(!done) == 0) break;
    }
    if (inside) accum[(size_t)py * W + px] = make_float4(cr + T * bg0, cg + T * bg1, cb + T * bg2, F_(1.0));
}

static cudaError_t grow(void** p, size_t& cap_bytes, size_t want) {
    if (*p && cap_bytes >= want) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    cap_bytes = 0;
    cudaError_t e = cudaMalloc(p, std::max<size_t>(want, 256));
    if (e == cudaSuccess) cap_bytes = std::max<size_t>(want, 256);
    return e;
}

void sorted_release(SortedState& s) {
    void* ptrs[] = {s.keys_a, s.vals_a, s.keys_b, s.vals_b, s.rec, s.tiles, s.cnt, s.scan_scratch,
                    s.ent_key_a, s.ent_val_a, s.ent_key_b, s.ent_val_b, s.ranges};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s.host_total) cudaFreeHost(s.host_total);
    radix_release(s.rs_keys);
    radix_release(s.rs_tiles);
    s = SortedState();
}

static cudaError_t exclusive_scan(SortedState& s, uint32_t* data, uint32_t n, uint32_t* total_dev, cudaStream_t st) {
    uint32_t nb = (n + kScTile - 1) / kScTile;
    if (nb > 1024u * 16u) return cudaErrorInvalidValue;
    cudaError_t e = grow(&s.scan_scratch, s.scan_scratch_bytes, ((size_t)nb + 64) * 4);
    if (e != cudaSuccess) return e;
    uint32_t* sums = (uint32_t*)s.scan_scratch;
    if (n == 0) return cudaMemsetAsync(total_dev, 0, 4, st);
    k_scan_reduce<<<nb, kScT, 0, st>>>(data, n, sums);
    k_scan_sums<<<1, 1024, 0, st>>>(sums, nb, total_dev);
    k_scan_apply<<<nb, kScT, 0, st>>>(data, n, sums);
    return cudaGetLastError();
}

cudaError_t sorted_render(SortedState& s, const FrameConst& f, const float4* splats, const float* sh, float4* accum,
                          unsigned long long* stats, uint32_t* err, int sm_count, bool full, cudaStream_t st,
                          std::string* what) {
    (void)sm_count;
    const uint32_t n = f.N;
    cudaError_t e;
    if (n > s.cap_n || !s.keys_a) {
        void** bufs[] = {&s.keys_a, &s.vals_a, &s.keys_b, &s.vals_b, &s.cnt};
        for (void** b : bufs) {
            if (*b) cudaFree(*b);
            *b = nullptr;
            if ((e = cudaMalloc(b, (size_t)std::max(n, 1u) * 4 + 64)) != cudaSuccess) { *what = "sorted buffers"; return e; }
        }
        if (s.rec) cudaFree(s.rec);
        if (s.tiles) cudaFree(s.tiles);
        s.rec = s.tiles = nullptr;
        if ((e = cudaMalloc(&s.rec, (size_t)std::max(n, 1u) * 48)) != cudaSuccess) { *what = "sorted records"; return e; }
        if ((e = cudaMalloc(&s.tiles, (size_t)std::max(n, 1u) * 8)) != cudaSuccess) { *what = "sorted rectangles"; return e; }
        if (!s.host_total && (e = cudaMallocHost(&s.host_total, 64)) != cudaSuccess) { *what = "pinned total"; return e; }
        s.cap_n = n;
    }
    TileGeom tg;
    tg.tw = s.tw;
    tg.th = s.th;
    tg.tiles_x = (f.W + tg.tw - 1) / tg.tw;
    tg.tiles_y = (f.H + tg.th - 1) / tg.th;
    cudaMemsetAsync(stats + ST_PROBE, 0, 8, st);  // the probe reports the last view (sorted.rs:316-322)
    k_sp_project<<<(n + 127) / 128, 128, 0, st>>>(f, tg, splats, sh, (uint32_t*)s.keys_a, (uint32_t*)s.vals_a,
                                                  (float4*)s.rec, (uint2*)s.tiles, stats, full ? 1 : 0);
    if ((e = cudaGetLastError()) != cudaSuccess) { *what = "sp_project kernel"; return e; }
    if (!full) return cudaSuccess;
    e = radix_sort_pairs(s.rs_keys, (uint32_t*)s.keys_a, (uint32_t*)s.vals_a, (uint32_t*)s.keys_b, (uint32_t*)s.vals_b, n, 24,
                         s.digit_bits, err, st);
    if (e != cudaSuccess) { *what = "depth sort"; return e; }
    k_gather_counts<<<(n + 255) / 256, 256, 0, st>>>((uint32_t*)s.keys_b, (uint32_t*)s.vals_b, (uint2*)s.tiles, n,
                                                     (uint32_t*)s.cnt);
    // total of tile entries: scan, then read it back to size the entry buffers
    e = grow(&s.scan_scratch, s.scan_scratch_bytes, ((size_t)((n + kScTile - 1) / kScTile) + 64) * 4);
    if (e != cudaSuccess) { *what = "scan scratch"; return e; }
    uint32_t nb = (n + kScTile - 1) / kScTile;
    uint32_t* total_dev = (uint32_t*)s.scan_scratch + nb + 16;
    if ((e = exclusive_scan(s, (uint32_t*)s.cnt, n, total_dev, st)) != cudaSuccess) { *what = "tile-count scan"; return e; }
    total_dev = (uint32_t*)s.scan_scratch + nb + 16;
    cudaMemcpyAsync(s.host_total, total_dev, 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) { *what = "sorted path"; return e; }
    uint32_t m = *(uint32_t*)s.host_total;
    uint32_t n_tiles = tg.tiles_x * tg.tiles_y;
    if (m > (1u << 30)) { *what = "more than 2^30 tile entries"; return cudaErrorInvalidValue; }
    if (m > s.cap_entries) {
        void** bufs[] = {&s.ent_key_a, &s.ent_val_a, &s.ent_key_b, &s.ent_val_b};
        size_t want = (size_t)m + m / 4 + 1024;
        for (void** b : bufs) {
            if (*b) cudaFree(*b);
            *b = nullptr;
            if ((e = cudaMalloc(b, want * 4)) != cudaSuccess) { *what = "tile entries"; return e; }
        }
        s.cap_entries = (uint32_t)want;
    }
    if (n_tiles > s.n_tiles || !s.ranges) {
        if (s.ranges) cudaFree(s.ranges);
        s.ranges = nullptr;
        if ((e = cudaMalloc(&s.ranges, (size_t)n_tiles * 8)) != cudaSuccess) { *what = "tile ranges"; return e; }
        s.n_tiles = n_tiles;
    }
    cudaMemsetAsync(s.ranges, 0, (size_t)n_tiles * 8, st);
    if (m) {
        k_emit_entries<<<(n + 255) / 256, 256, 0, st>>>((uint32_t*)s.keys_b, (uint32_t*)s.vals_b, (uint2*)s.tiles,
                                                        (uint32_t*)s.cnt, n, tg.tiles_x, (uint32_t*)s.ent_key_a,
                                                        (uint32_t*)s.ent_val_a);
        int tbits = 1;
        while ((1u << tbits) < n_tiles) ++tbits;
        e = radix_sort_pairs(s.rs_tiles, (uint32_t*)s.ent_key_a, (uint32_t*)s.ent_val_a, (uint32_t*)s.ent_key_b,
                             (uint32_t*)s.ent_val_b, m, tbits, 8, err, st);
        if (e != cudaSuccess) { *what = "tile sort"; return e; }
        k_tile_ranges<<<(m + 255) / 256, 256, 0, st>>>((uint32_t*)s.ent_key_b, m, (uint2*)s.ranges);
    }
    if (s.tw == 16 && s.th == 16)
        k_blend<16, 16><<<n_tiles, 256, 0, st>>>(f.W, f.H, tg.tiles_x, (uint2*)s.ranges, (uint32_t*)s.ent_val_b,
                                                 (uint32_t*)s.vals_b, (float4*)s.rec, f.bg[0], f.bg[1], f.bg[2], accum);
    else if (s.tw == 32 && s.th == 8)
        k_blend<32, 8><<<n_tiles, 256, 0, st>>>(f.W, f.H, tg.tiles_x, (uint2*)s.ranges, (uint32_t*)s.ent_val_b,
                                                (uint32_t*)s.vals_b, (float4*)s.rec, f.bg[0], f.bg[1], f.bg[2], accum);
    else
        k_blend<32, 32><<<n_tiles, 1024, 0, st>>>(f.W, f.H, tg.tiles_x, (uint2*)s.ranges, (uint32_t*)s.ent_val_b,
                                                  (uint32_t*)s.vals_b, (float4*)s.rec, f.bg[0], f.bg[1], f.bg[2], accum);
    if ((e = cudaGetLastError()) != cudaSuccess) { *what = "blend kernel"; return e; }
    return cudaSuccess;
}

cudaError_t sorted_read(SortedState& s, uint32_t* keys, uint32_t* vals, uint32_t n, cudaStream_t st) {
    if (!s.keys_b || n > s.cap_n) return cudaErrorInvalidValue;
    cudaMemcpyAsync(keys, s.keys_b, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(vals, s.vals_b, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    return cudaStreamSynchronize(st);
}

// ============================================================================ composite
__device__ __forceinline__ float oetf(float c) {
    if (c <= F_(0.0031308)) return F_(12.92) * c;
    return F_(1.055) * gx::pow(c, gxc::kInv2p4) - F_(0.055);
}
__device__ __forceinline__ void lin_px(const float4* accum, uint32_t W, uint32_t H, int px, int py, float* c) {
    int qx = min(max(px, 0), (int)W - 1), qy = min(max(py, 0), (int)H - 1);
    float4 a = __ldg(&accum[(size_t)qy * W + qx]);
    float d = fmax_(a.w, F_(1.0));
    c[0] = div_(a.x, d);
    c[1] = div_(a.y, d);
    c[2] = div_(a.z, d);
}
__device__ __forceinline__ float mixc(float a, float b, float t) { return a * (F_(1.0) - t) + b * t; }

__global__ void k_composite(const float4* __restrict__ accum, uint32_t W, uint32_t H, float exposure, uint32_t gamma_on,
                            uint32_t out_w, uint32_t out_h, uchar4* out) {
    uint32_t X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y;
    if (X >= out_w || Y >= out_h) return;
    float uvx = div_((float)X + F_(0.5), (float)out_w), uvy = div_((float)Y + F_(0.5), (float)out_h);
    float qx = uvx * (float)W - F_(0.5), qy = uvy * (float)H - F_(0.5);
    float fx0 = floorf(qx), fy0 = floorf(qy);
    int px = (int)fx0, py = (int)fy0;
    float fx = qx - fx0, fy = qy - fy0;
    float c00[3], c10[3], c01[3], c11[3];
    lin_px(accum, W, H, px, py, c00);
    lin_px(accum, W, H, px + 1, py, c10);
    lin_px(accum, W, H, px, py + 1, c01);
    lin_px(accum, W, H, px + 1, py + 1, c11);
    unsigned char o[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float top = mixc(c00[k], c10[k], fx), bot = mixc(c01[k], c11[k], fx);
        float c = mixc(top, bot, fy) * exposure;
        c = clamp_(c, F_(0.0), F_(1.0));
        if (gamma_on) c = oetf(c);
        o[k] = (unsigned char)f2u(gx::rint_(c * F_(255.0)));
    }
    out[(size_t)Y * out_w + X] = make_uchar4(o[0], o[1], o[2], 255);
}

void launch_composite(const float4* accum, uint32_t W, uint32_t H, float exposure, uint32_t gamma_on, uint32_t out_w,
                      uint32_t out_h, uchar4* out, cudaStream_t st) {
    dim3 grid((out_w + 255) / 256, out_h);
    k_composite<<<grid, 256, 0, st>>>(accum, W, H, exposure, gamma_on, out_w, out_h, out);
}

}  // namespace gpsb

// ============================================================================ C ABI: no-allocation sort
namespace gpsb {
void set_global_error(const char* msg);  // renderer.cpp: message of gpsb_last_error(NULL)
}
static thread_local char g_noalloc_error[256];

extern "C" gpsb_status gpsb_sort_pairs_noalloc(uint32_t* keys_in, uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                                               uint32_t n, uint32_t key_bits, void* cuda_stream, uint32_t* err_dev) {
    using namespace gpsb;
    g_noalloc_error[0] = 0;
    if (n > kNoAllocMaxN) {
        snprintf(g_noalloc_error, sizeof g_noalloc_error,
                 "gpsb_sort_pairs_noalloc: %u pairs exceed the fixed scratch of %u pairs", n, kNoAllocMaxN);
        set_global_error(g_noalloc_error);
        return GPSB_ERR_LIMIT;
    }
    if (key_bits < 1 || key_bits > 32) {
        snprintf(g_noalloc_error, sizeof g_noalloc_error, "gpsb_sort_pairs_noalloc: key_bits must be 1..32");
        set_global_error(g_noalloc_error);
        return GPSB_ERR_INVALID_ARGUMENT;
    }
    if (n == 0) return GPSB_OK;
    if (!keys_in || !vals_in || !keys_out || !vals_out || !err_dev) {
        snprintf(g_noalloc_error, sizeof g_noalloc_error, "gpsb_sort_pairs_noalloc: null buffer or error word");
        set_global_error(g_noalloc_error);
        return GPSB_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = (cudaStream_t)cuda_stream;
    cudaError_t e;
    bool capture_without_setup = false;
    uint32_t* base = (uint32_t*)noalloc_scratch_address(st, &e, &capture_without_setup);
    if (!base) {
        if (capture_without_setup)
            snprintf(g_noalloc_error, sizeof g_noalloc_error,
                     "gpsb_sort_pairs_noalloc: the first call on a device must come before any stream capture");
        else
            snprintf(g_noalloc_error, sizeof g_noalloc_error, "gpsb_sort_pairs_noalloc: scratch address: %s",
                     cudaGetErrorString(e));
        set_global_error(g_noalloc_error);
        return capture_without_setup ? GPSB_ERR_STATE : GPSB_ERR_CUDA;
    }
    const int passes = (int)((key_bits + 7) / 8);
    const uint32_t tiles = (n + RsShape<8>::tile - 1) / RsShape<8>::tile;
    uint32_t* hist = base;
    uint32_t* counters = base + kNoAllocHistWords;
    uint32_t* err = err_dev;
    uint32_t* lookback = base + kNoAllocHistWords + kNoAllocCounterWords;
    // the array keeps the previous call's contents: clear what this call needs at zero
    e = cudaMemsetAsync(base, 0, (kNoAllocHistWords + kNoAllocCounterWords) * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(lookback, 0, (size_t)passes * tiles * 256 * 4, st);
    uint32_t *ik = keys_in, *iv = vals_in, *ok = keys_out, *ov = vals_out;
    if (e == cudaSuccess && passes % 2 == 0) {
        // an even number of passes ends in the first buffer: start from a copy in the output
        e = cudaMemcpyAsync(keys_out, keys_in, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(vals_out, vals_in, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
        ik = keys_out; iv = vals_out; ok = keys_in; ov = vals_in;
    }
    if (e == cudaSuccess) {
        k_radix_hist<8><<<std::min<uint32_t>((n + 4095) / 4096, 1184u), 256, 0, st>>>(ik, n, passes, hist);
        k_radix_hist_scan<8><<<1, 32, 0, st>>>(hist, passes);
        for (int p = 0; p < passes; ++p) {
            onesweep_launch<8>(tiles, ik, iv, ok, ov, n, p * 8, hist + p * 256, lookback + (size_t)p * tiles * 256,
                               counters + p, err, st);
            std::swap(ik, ok);
            std::swap(iv, ov);
        }
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        snprintf(g_noalloc_error, sizeof g_noalloc_error, "gpsb_sort_pairs_noalloc: %s", cudaGetErrorString(e));
        set_global_error(g_noalloc_error);
        return GPSB_ERR_CUDA;
    }
    return GPSB_OK;
}
