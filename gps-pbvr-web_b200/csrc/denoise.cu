// Kernels of the learned denoiser: 3x3 convolutions (stride 1, zero padding 1) over NHWC bf16
// activations as implicit GEMMs on the tcgen05 engine of umma.cuh, their weight gradients, and
// the element-wise steps of the U-Net (ReLU backward, 2x2 average pooling, nearest upsampling,
// L1 loss, Adam). Channel counts are padded to multiples of 8 so that every 16-byte chunk of an
// activation row holds 8 channels of one pixel.
//
//   forward   Y[p][n]  = act(bias[n] + sum_k Xcol[p][k] W[n][k]),  k = (ky*3 + kx)*Cin + ci
//   data grad dX       = the forward convolution of dY with W'[ci][(2-ky)*3 + (2-kx)][co] = W[co][ky*3+kx][ci]
//   weight grad dW[n][k] = sum_p dY[p][n] Xcol[p][k]  (rows n, split over pixel ranges, fp32 atomics)
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "umma.cuh"

namespace gpsb {
namespace dn {

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------------------- implicit-im2col conv
struct ConvFwd {
    const bf16* x;      // [B][H][W][ldx], input channels at offset xoff
    int ldx, xoff, cin; // cin: multiple of 8
    int B, H, W;
    const bf16* w;      // [cout][kp] (K-major, zero past 9*cin)
    int cout, kp;
    const float* bias;  // [cout] or null
    void* out;          // [B*H*W][ldo] at channel offset ooff: bf16, or fp32 when out_f32
    int ldo, ooff, out_f32, relu;
    uint32_t* err;

    __device__ __forceinline__ void load_a(uint8_t* tile, int m0, int k0) const {
        const int M = B * H * W, K = 9 * cin;
#pragma unroll 2
        for (int c = threadIdx.x; c < umma::kBM * 8; c += umma::kThreads) {
            const int r8 = c & 7, kc = (c >> 3) & 7, rg = c >> 6;
            const int row = rg * 8 + r8, m = m0 + row, k = k0 + kc * 8;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (m < M && k < K) {
                const int tap = k / cin, ci = k - tap * cin;
                const int xq = m % W, yq = (m / W) % H, b = m / (W * H);
                const int yy = yq + tap / 3 - 1, xx = xq + tap % 3 - 1;
                if (yy >= 0 && yy < H && xx >= 0 && xx < W)
                    v = __ldg(reinterpret_cast<const uint4*>(x + ((size_t)(b * H + yy) * W + xx) * ldx + xoff + ci));
            }
            *reinterpret_cast<uint4*>(tile + c * 16) = v;
        }
    }
    template <int BN>
    __device__ __forceinline__ void load_b_t(uint8_t* tile, int n0, int k0) const {
        for (int c = threadIdx.x; c < BN * 8; c += umma::kThreads) {
            const int r8 = c & 7, kc = (c >> 3) & 7, rg = c >> 6;
            const int n = n0 + rg * 8 + r8, k = k0 + kc * 8;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (n < cout && k < kp) v = __ldg(reinterpret_cast<const uint4*>(w + (size_t)n * kp + k));
            *reinterpret_cast<uint4*>(tile + c * 16) = v;
        }
    }
    __device__ __forceinline__ void epilogue(int m0, int n0, int row, int col0, const float* v) const {
        const int m = m0 + row;
        if (m >= B * H * W) return;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int n = n0 + col0 + j;
            if (n >= cout) break;
            float y = v[j] + (bias ? bias[n] : 0.0f);
            if (relu) y = fmaxf(y, 0.0f);
            const size_t o = (size_t)m * ldo + ooff + n;
            if (out_f32) reinterpret_cast<float*>(out)[o] = y;
            else reinterpret_cast<bf16*>(out)[o] = __float2bfloat16_rn(y);
        }
    }
};

template <int BN>
struct ConvFwdN : ConvFwd {
    __device__ __forceinline__ void load_b(uint8_t* tile, int n0, int k0) const { load_b_t<BN>(tile, n0, k0); }
};

template <int BN>
__global__ void __launch_bounds__(umma::kThreads) k_conv_fwd(ConvFwdN<BN> pb) {
    umma::gemm_tile<BN>(pb, blockIdx.x * umma::kBM, blockIdx.y * BN, 0, pb.kp);
}

// ---------------------------------------------------------------------------- weight gradient
// 8x8 transpose of bf16 values: in[p] holds 8 channels of pixel p, out[c] 8 pixels of channel c
__device__ __forceinline__ void transpose8(const uint4* in, uint4* out) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(in);  // w[p*4 + j] = channels (2j, 2j+1) of pixel p
    uint32_t* o = reinterpret_cast<uint32_t*>(out);             // o[c*4 + i] = pixels (2i, 2i+1) of channel c
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t a = w[(2 * i) * 4 + j], b = w[(2 * i + 1) * 4 + j];
            o[(2 * j) * 4 + i] = __byte_perm(a, b, 0x5410);
            o[(2 * j + 1) * 4 + i] = __byte_perm(a, b, 0x7632);
        }
}

struct ConvDW {
    const bf16* dy;     // [M][ldy] output gradient (bf16), cout channels at offset 0
    int ldy;
    const bf16* x;      // layer input [M][ldx] at channel offset xoff, cin channels
    int ldx, xoff, cin;
    int B, H, W;
    int cout, kp;
    float* dw;          // [cout][kp] fp32, accumulated with atomics
    int pix_per_cta;    // multiple of 64
    uint32_t* err;

    // rows = output channels (128, zero past cout), 64 pixels: one 8-channel x 8-pixel block per thread
    __device__ __forceinline__ void load_a(uint8_t* tile, int m0, int p0) const {
        const int M = B * H * W;
        const int cg = threadIdx.x >> 3, pg = threadIdx.x & 7;  // 16 channel groups x 8 pixel groups
        uint4 in[8], out[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int p = p0 + pg * 8 + q, c = m0 + cg * 8;
            in[q] = (p < M && c < cout) ? __ldg(reinterpret_cast<const uint4*>(dy + (size_t)p * ldy + c))
                                        : make_uint4(0u, 0u, 0u, 0u);
        }
        transpose8(in, out);
#pragma unroll
        for (int r = 0; r < 8; ++r) *reinterpret_cast<uint4*>(tile + umma::chunk_off(cg * 8 + r, pg)) = out[r];
    }
    template <int BN>
    __device__ __forceinline__ void load_b_t(uint8_t* tile, int n0, int p0) const {
        const int M = B * H * W, K = 9 * cin;
        for (int blk = threadIdx.x; blk < (BN / 8) * 8; blk += umma::kThreads) {
            const int kg = blk >> 3, pg = blk & 7;
            const int k = n0 + kg * 8;
            uint4 in[8], out[8];
            const bool kok = k < K;
            const int tap = kok ? k / cin : 0, ci = kok ? k - tap * cin : 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int p = p0 + pg * 8 + q;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (kok && p < M) {
                    const int xq = p % W, yq = (p / W) % H, b = p / (W * H);
                    const int yy = yq + tap / 3 - 1, xx = xq + tap % 3 - 1;
                    if (yy >= 0 && yy < H && xx >= 0 && xx < W)
                        v = __ldg(reinterpret_cast<const uint4*>(x + ((size_t)(b * H + yy) * W + xx) * ldx + xoff + ci));
                }
                in[q] = v;
            }
            transpose8(in, out);
#pragma unroll
            for (int r = 0; r < 8; ++r) *reinterpret_cast<uint4*>(tile + umma::chunk_off(kg * 8 + r, pg)) = out[r];
        }
    }
    __device__ __forceinline__ void epilogue(int m0, int n0, int row, int col0, const float* v) const {
        const int co = m0 + row;
        if (co >= cout) return;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int k = n0 + col0 + j;
            if (k < 9 * cin && v[j] != 0.0f) atomicAdd(&dw[(size_t)co * kp + k], v[j]);
        }
    }
};

template <int BN>
struct ConvDWN : ConvDW {
    __device__ __forceinline__ void load_b(uint8_t* tile, int n0, int k0) const { load_b_t<BN>(tile, n0, k0); }
};

template <int BN>
__global__ void __launch_bounds__(umma::kThreads) k_conv_dw(ConvDWN<BN> pb) {
    const int M = pb.B * pb.H * pb.W;
    const int p_begin = blockIdx.y * pb.pix_per_cta;
    int p_end = p_begin + pb.pix_per_cta;
    const int mpad = (M + 63) / 64 * 64;
    if (p_end > mpad) p_end = mpad;
    if (p_begin >= p_end) return;
    umma::gemm_tile<BN>(pb, 0, blockIdx.x * BN, p_begin, p_end);
}

// ---------------------------------------------------------------------------- weight flip
// W'[ci][t'][co] = W[co][8 - t'][ci] for the data gradient; W' rows padded to kp2 = 9 * coutp (64-multiple)
__global__ void k_flip(const bf16* w, int cout, int cin, int kp, bf16* wf, int coutp, int kp2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // over cin * kp2
    if (i >= cin * kp2) return;
    const int ci = i / kp2, k2 = i - ci * kp2;
    bf16 v = __float2bfloat16_rn(0.0f);
    if (k2 < 9 * coutp) {
        const int t2 = k2 / coutp, co = k2 - t2 * coutp;
        if (co < cout) v = w[(size_t)co * kp + (8 - t2) * cin + ci];
    }
    wf[i] = v;
}

}  // namespace dn
}  // namespace gpsb

using namespace gpsb;
using namespace gpsb::dn;

template <int BN>
static cudaError_t launch_fwd(const ConvFwd& p, cudaStream_t st) {
    ConvFwdN<BN> q;
    static_cast<ConvFwd&>(q) = p;
    const size_t smem = umma::smem_bytes<BN>();
    cudaFuncSetAttribute(k_conv_fwd<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int M = p.B * p.H * p.W;
    dim3 grid((M + umma::kBM - 1) / umma::kBM, (p.cout + BN - 1) / BN);
    k_conv_fwd<BN><<<grid, umma::kThreads, smem, st>>>(q);
    return cudaGetLastError();
}

template <int BN>
static cudaError_t launch_dw(const ConvDW& p, cudaStream_t st) {
    ConvDWN<BN> q;
    static_cast<ConvDW&>(q) = p;
    const size_t smem = umma::smem_bytes<BN>();
    cudaFuncSetAttribute(k_conv_dw<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int M = p.B * p.H * p.W;
    dim3 grid((9 * p.cin + BN - 1) / BN, (M + p.pix_per_cta - 1) / p.pix_per_cta);
    k_conv_dw<BN><<<grid, umma::kThreads, smem, st>>>(q);
    return cudaGetLastError();
}

extern "C" {

// 3x3 convolution, stride 1, zero padding 1, NHWC bf16 in, bf16 or fp32 out (see ConvFwd).
// Returns a cudaError_t code (0 = launched).
int gpsb_dn_conv_fwd(const void* x, int ldx, int xoff, int cin, int B, int H, int W, const void* w, int cout, int kp,
                     const float* bias, void* out, int ldo, int ooff, int out_f32, int relu, void* stream,
                     uint32_t* err) {
    if (cin % 8 || ldx % 8 || xoff % 8 || kp % 64 || kp < 9 * cin || cout < 1 || cout > 256) return (int)cudaErrorInvalidValue;
    ConvFwd p{(const bf16*)x, ldx, xoff, cin, B, H, W, (const bf16*)w, cout, kp, bias, out, ldo, ooff, out_f32, relu, err};
    cudaStream_t st = (cudaStream_t)stream;
    if (cout <= 16) return (int)launch_fwd<16>(p, st);
    if (cout <= 32) return (int)launch_fwd<32>(p, st);
    if (cout <= 64) return (int)launch_fwd<64>(p, st);
    if (cout <= 128) return (int)launch_fwd<128>(p, st);
    return (int)launch_fwd<256>(p, st);
}

// Weight gradient dw[co][k] += sum_p dy[p][co] * xcol[p][k] (fp32 accumulate into dw, which the
// caller zeroes); cout <= 128, dy channels padded to a multiple of 8.
int gpsb_dn_conv_dw(const void* dy, int ldy, const void* x, int ldx, int xoff, int cin, int B, int H, int W, int cout,
                    int kp, float* dw, void* stream, uint32_t* err) {
    if (cin % 8 || ldx % 8 || xoff % 8 || ldy % 8 || kp < 9 * cin || cout < 1 || cout > 128) return (int)cudaErrorInvalidValue;
    const int M = B * H * W;
    // about four CTAs per SM over the pixel splits and the K tiles
    const int ktiles = (9 * cin + 127) / 128;
    int splits = (148 * 4 + ktiles - 1) / ktiles;
    int ppc = (M + splits - 1) / splits;
    ppc = (ppc + 63) / 64 * 64;
    if (ppc < 256) ppc = 256;
    ConvDW p{(const bf16*)dy, ldy, (const bf16*)x, ldx, xoff, cin, B, H, W, cout, kp, dw, ppc, err};
    return (int)launch_dw<128>(p, (cudaStream_t)stream);
}

// W' for the data gradient (see k_flip); wf is [cin][kp2], kp2 >= 9 * coutp, a multiple of 64.
int gpsb_dn_flip(const void* w, int cout, int cin, int kp, void* wf, int coutp, int kp2, void* stream) {
    if (kp2 % 64 || kp2 < 9 * coutp || coutp < cout) return (int)cudaErrorInvalidValue;
    const int n = cin * kp2;
    k_flip<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>((const bf16*)w, cout, cin, kp, (bf16*)wf, coutp, kp2);
    return (int)cudaGetLastError();
}

}  // extern "C"
