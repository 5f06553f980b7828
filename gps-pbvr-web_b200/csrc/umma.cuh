// Tensor-core GEMM engine for sm_100a (5th-generation tensor cores, tcgen05): the building block of
// the denoiser's convolutions. One CTA of 128 threads computes a 128 x BN tile of
//     C[m][n] = sum_k A[m][k] * B[n][k]        (A, B bf16, accumulation in fp32 in tensor memory)
// over the K range [k_begin, k_end), in steps of 64. Operand tiles are staged in shared memory by
// all threads through problem-specific loaders (implicit im2col, transposing gathers), in the
// canonical K-major layout without swizzle: core matrices of 8 rows x 16 bytes, row group rg and
// 8-element K chunk kc at byte (rg * 8 + kc) * 128, so the K-adjacent core matrices of one MMA
// are 128 bytes apart (leading byte offset) and the next 8 rows 1024 bytes (stride byte offset).
// Two stages: while the tensor core multiplies one stage, the threads fill the other. Thread 0
// issues the MMAs (M = 128, N = BN, K = 16 each) and commits them to an mbarrier per stage; the
// accumulator (128 lanes x BN fp32 columns of tensor memory) is read back by the four warps with
// tcgen05.ld (warp w owns lanes 32w..32w+31 = tile rows) and handed to the problem's epilogue.
// Every wait is bounded; on a timeout the CTA records GEMM_ERR_TIMEOUT, waits (bounded) for its
// MMAs, frees its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace gpsb {
namespace umma {

constexpr int kThreads = 128;
constexpr int kBM = 128;
constexpr int kBK = 64;
constexpr uint32_t kSpin = 1u << 24;
constexpr uint32_t GEMM_ERR_TIMEOUT = 8u;

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of the 16-byte chunk (row, kc) inside a K-major no-swizzle tile
__device__ __forceinline__ uint32_t chunk_off(uint32_t row, uint32_t kc) {
    return ((row >> 3) * 8u + kc) * 128u + (row & 7u) * 16u;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    const uint64_t lbo = 128, sbo = 1024;
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((lbo >> 4) << 16) | ((sbo >> 4) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: D fp32, A and B bf16, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < kSpin; ++i)
        if (mbar_test(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive fp32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// The same load without the wait: several loads can be in flight before one tmem_ld_wait(), after
// which (and not before) v holds the columns.
__device__ __forceinline__ void tmem_ld16_issue(uint32_t taddr, float* v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]),
          "=f"(v[8]), "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15])
        : "r"(taddr)
        : "memory");
}
// Waits for this thread's tensor-memory loads; every register of v is passed through an empty asm
// after the wait, so the compiler can schedule no use of a loaded value before it.
template <int n>
__device__ __forceinline__ void tmem_ld_wait(float (&v)[n]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < n; ++i) asm volatile("" : "+f"(v[i]));
}

template <int BN>
__host__ __device__ constexpr uint32_t tmem_cols() {
    return BN <= 32 ? 32u : BN <= 64 ? 64u : BN <= 128 ? 128u : 256u;
}
template <int BN>
__host__ __device__ constexpr size_t smem_bytes() {
    return 2 * ((size_t)kBM * kBK * 2 + (size_t)BN * kBK * 2) + 128;
}

// The GEMM mainloop. P provides:
//   __device__ void load_a(uint8_t* tile, int m0, int k0) const   // 128 x 64 bf16 K-major tile
//   __device__ void load_b(uint8_t* tile, int n0, int k0) const   // BN x 64
//   __device__ void epilogue(int m0, int n0, int row, int col0, const float* v16) const
//   int k_begin, k_end (multiples of 64), m0/n0 from the grid via tile(), err (uint32_t*)
template <int BN, class P>
__device__ __forceinline__ void gemm_tile(const P& pb, int m0, int n0, int k_begin, int k_end) {
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "N of one MMA");
    extern __shared__ __align__(128) uint8_t s_raw[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(s_raw) + 127) & ~(uintptr_t)127);
    constexpr uint32_t kABytes = kBM * kBK * 2, kBBytes = BN * kBK * 2;
    auto sa = [&](int b) { return base + b * kABytes; };
    auto sb = [&](int b) { return base + 2 * kABytes + b * kBBytes; };
    const int tid = threadIdx.x, warp = tid >> 5;
    constexpr uint32_t kCols = tmem_cols<BN>();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&s_tmem)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&s_bar[0]);
        mbar_init(&s_bar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    const int steps = (k_end - k_begin) / kBK;
    if (steps > 0) {
        pb.load_a(sa(0), m0, k_begin);
        pb.load_b(sb(0), n0, k_begin);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = s_tmem;
    constexpr uint32_t idesc = idesc_bf16(BN);
    for (int s = 0; s < steps; ++s) {
        const int buf = s & 1;
        if (tid == 0) {
            const uint32_t a0 = saddr(sa(buf)), b0 = saddr(sb(buf));
#pragma unroll
            for (int j = 0; j < kBK / 16; ++j)  // K = 16 = two core matrices = 256 bytes per MMA
                mma_bf16(tmem, smem_desc(a0 + j * 256), smem_desc(b0 + j * 256), idesc, s > 0 || j > 0);
            mma_commit(&s_bar[buf]);
        }
        if (s + 1 < steps) {
            if (s >= 1 && !mbar_wait(&s_bar[buf ^ 1], ((s - 1) >> 1) & 1)) s_fail = 1;
            pb.load_a(sa(buf ^ 1), m0, k_begin + (s + 1) * kBK);
            pb.load_b(sb(buf ^ 1), n0, k_begin + (s + 1) * kBK);
            fence_async_smem();
        }
        fence_before();
        __syncthreads();
        fence_after();
        if (s_fail) break;
    }
    bool ok = !s_fail;
    if (steps > 0 && ok) ok = mbar_wait(&s_bar[(steps - 1) & 1], ((steps - 1) >> 1) & 1);
    if (!ok) {
        if (tid == 0) atomicOr(pb.err, GEMM_ERR_TIMEOUT);
        // let every MMA this CTA issued finish before its tensor memory is freed
        if (steps > 0) mbar_wait(&s_bar[(steps - 1) & 1], ((steps - 1) >> 1) & 1);
    }
    fence_after();
    if (ok && steps > 0) {
        const int row = warp * 32 + (tid & 31);
#pragma unroll 1
        for (int c = 0; c < BN; c += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
            pb.epilogue(m0, n0, row, c, v);
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

// Issue one asynchronous 16-byte global -> shared copy; bytes < 16 zero-fills the rest (0: all zero).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr(dst)), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <int BN, int S>
__host__ __device__ constexpr size_t smem_bytes_async() {
    return (size_t)S * ((size_t)kBM * kBK * 2 + (size_t)BN * kBK * 2) + 128;
}

// The mainloop with S stages filled by asynchronous copies: P provides
//   __device__ void prepare(int m0, int n0)                   // per-tile loader state (registers)
//   __device__ void issue(uint8_t* a_tile, uint8_t* b_tile, int k0)   // cp.async of one K step
//   __device__ void epilogue(...), err    (as gemm_tile)
// Stage s is copied S-1 steps ahead; a stage is refilled only after the MMAs that read it have
// completed (their mbarrier), and the tensor core reads a stage only after every thread's copies
// into it have landed (cp.async.wait_group + proxy fence + barrier).
template <int BN, int S, class P>
__device__ __forceinline__ void gemm_tile_async(P& pb, int m0, int n0, int k_begin, int k_end) {
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256 && S >= 2 && S <= 6, "shape");
    extern __shared__ __align__(128) uint8_t s_raw[];
    __shared__ __align__(8) uint64_t s_bar[S];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(s_raw) + 127) & ~(uintptr_t)127);
    constexpr uint32_t kABytes = kBM * kBK * 2, kBBytes = BN * kBK * 2;
    auto sa = [&](int b) { return base + b * kABytes; };
    auto sb = [&](int b) { return base + S * kABytes + b * kBBytes; };
    const int tid = threadIdx.x, warp = tid >> 5;
    constexpr uint32_t kCols = tmem_cols<BN>();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&s_tmem)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < S; ++i) mbar_init(&s_bar[i]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    pb.prepare(m0, n0);
    const int steps = (k_end - k_begin) / kBK;
#pragma unroll
    for (int i = 0; i < S - 1; ++i) {
        if (i < steps) pb.issue(sa(i), sb(i), k_begin + i * kBK);
        cp_async_commit();
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = s_tmem;
    constexpr uint32_t idesc = idesc_bf16(BN);
    for (int s = 0; s < steps; ++s) {
        const int buf = s % S;
        cp_async_wait<S - 2>();  // this thread's copies of stage s have landed
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        if (s_fail) break;
        if (tid == 0) {
            const uint32_t a0 = saddr(sa(buf)), b0 = saddr(sb(buf));
#pragma unroll
            for (int j = 0; j < kBK / 16; ++j)
                mma_bf16(tmem, smem_desc(a0 + j * 256), smem_desc(b0 + j * 256), idesc, s > 0 || j > 0);
            mma_commit(&s_bar[buf]);
        }
        // refill the stage read by step s-1 with step s+S-1, once those MMAs are done
        const int nxt = s + S - 1;
        if (nxt < steps) {
            const int nb = nxt % S;
            if (s >= 1 && !mbar_wait(&s_bar[nb], ((s - 1) / S) & 1)) s_fail = 1;
            pb.issue(sa(nb), sb(nb), k_begin + nxt * kBK);
        }
        cp_async_commit();
    }
    cp_async_wait<0>();
    bool ok = !s_fail;
    const int last = steps - 1;
    if (steps > 0 && ok) ok = mbar_wait(&s_bar[last % S], (last / S) & 1);
    if (!ok) {
        if (tid == 0) atomicOr(pb.err, GEMM_ERR_TIMEOUT);
        if (steps > 0) mbar_wait(&s_bar[last % S], (last / S) & 1);
    }
    fence_after();
    if (ok && steps > 0) {
        const int row = warp * 32 + (tid & 31);
#pragma unroll 1
        for (int c = 0; c < BN; c += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
            pb.epilogue(m0, n0, row, c, v);
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

}  // namespace umma
}  // namespace gpsb
