// Kernels of the learned denoiser: 3x3 convolutions (stride 1, zero padding 1) as implicit GEMMs on
// the tcgen05 engine of umma.cuh (the earlier engine, pixel-major NHWC in and out), the weight
// gradients, and the element-wise steps of the U-Net (ReLU backward, 2x2 average pooling, nearest
// upsampling, L1 loss, Adam). The network's bf16 activations are chunk-planar, [B][C/8][H][W][8]
// (the layout conv3x3.cu reads with TMA); its fp32 buffers (gradients, residual) are pixel-major.
// Channel counts are padded to multiples of 8; an 8-channel tensor is the same in both layouts.
//
//   forward   Y[p][n]  = act(bias[n] + sum_k Xcol[p][k] W[n][k]),  k = (ky*3 + kx)*Cin + ci
//   data grad dX       = the forward convolution of dY with W'[ci][(2-ky)*3 + (2-kx)][co] = W[co][ky*3+kx][ci]
//   weight grad dW[n][k] = sum_p dY[p][n] Xcol[p][k]  (rows n, split over pixel ranges, fp32 atomics)
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "pdl.cuh"
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

// Asynchronous loader of the forward convolution: every thread owns 8 rows (pixels) of the A tile
// and one 8-channel chunk column per K step; the pixels' coordinates are decoded once per tile and
// each 16-byte chunk is a cp.async with zero fill (src-size 0) for padding taps and tails.
template <int BN>
struct ConvFwdN : ConvFwd {
    int pix[8], py[8], px[8];

    __device__ __forceinline__ void prepare(int m0, int) {
        const int M = B * H * W, tid = threadIdx.x;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int row = 8 * ((tid >> 6) + 2 * i) + (tid & 7), m = m0 + row;
            pix[i] = m;
            if (m < M) {
                px[i] = m % W;
                py[i] = (m / W) % H;
            } else {
                px[i] = 0;
                py[i] = -4;  // never inside the image
            }
        }
    }
    __device__ __forceinline__ void issue(uint8_t* a_tile, uint8_t* b_tile, int k0) const {
        const int tid = threadIdx.x, K = 9 * cin;
        const int k = k0 + ((tid >> 3) & 7) * 8;
        const bool kok = k < K;
        const int tap = kok ? k / cin : 0, ci = k - tap * cin;
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int yy = py[i] + dy, xx = px[i] + dx;
            const bool ok = kok && yy >= 0 && yy < H && xx >= 0 && xx < W;
            const bf16* src = ok ? x + (size_t)(pix[i] + dy * W + dx) * ldx + xoff + ci : x;
            umma::cp_async16(a_tile + (tid + umma::kThreads * i) * 16, src, ok ? 16u : 0u);
        }
        for (int c = tid; c < BN * 8; c += umma::kThreads) {
            const int n = n0_ + (c >> 6) * 8 + (c & 7), kk = k0 + ((c >> 3) & 7) * 8;
            const bool ok = n < cout && kk < kp;
            umma::cp_async16(b_tile + c * 16, ok ? w + (size_t)n * kp + kk : w, ok ? 16u : 0u);
        }
    }
    int n0_ = 0;
};

// Pipeline stages of the forward convolution: the short K loops (2-14 steps of 64) gain more from
// resident CTAs than from deep pipelines; 1280x720 inference 4.33 ms with 4 / 3 stages, 3.99 ms
// with 2 / 3, 4.07 with 2 / 2, 4.09 with 3 / 2
#ifndef GPSB_CONV_STAGES
#define GPSB_CONV_STAGES 2  // below 128 output channels
#endif
#ifndef GPSB_CONV_STAGES_WIDE
#define GPSB_CONV_STAGES_WIDE 3  // ... and at 128
#endif
template <int BN>
__host__ __device__ constexpr int fwd_stages() { return BN >= 128 ? GPSB_CONV_STAGES_WIDE : GPSB_CONV_STAGES; }

template <int BN>
__global__ void __launch_bounds__(umma::kThreads) k_conv_fwd(ConvFwdN<BN> pb) {
    ConvFwdN<BN> q = pb;
    q.n0_ = blockIdx.y * BN;
    umma::gemm_tile_async<BN, fwd_stages<BN>()>(q, blockIdx.x * umma::kBM, blockIdx.y * BN, 0, pb.kp);
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
    const bf16* dy;     // output gradient, chunk-planar of ldy channels (bf16), cout channels at offset 0
    int ldy;
    const bf16* x;      // layer input, chunk-planar of ldx channels, cin channels at offset xoff
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
            const int HW = H * W, b = p / HW, pix = p - b * HW;
            in[q] = (p < M && c < cout)
                        ? __ldg(reinterpret_cast<const uint4*>(dy + (((size_t)b * (ldy / 8) + c / 8) * HW + pix) * 8))
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
                        v = __ldg(reinterpret_cast<const uint4*>(
                            x + ((((size_t)b * (ldx / 8) + (xoff + ci) / 8) * H + yy) * W + xx) * 8));
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


// ---------------------------------------------------------------------------- element-wise steps
__device__ __forceinline__ int gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }

// out (chunk-planar, ldo channels, B images of HW pixels): channel c < C = g[pix][goff + c] (fp32
// pixel-major) masked by y[pix][yoff + c] > 0 (chunk-planar, y null: no mask), 0 for C <= c < ldo
__global__ void k_relu_bwd(const float* g, int ldg, int goff, const bf16* y, int ldy, int yoff, int B, int HW, int C,
                           bf16* out, int ldo) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)B * HW * ldo) return;
    const int e = (int)(i & 7);
    long t = i >> 3;
    const int pix = (int)(t % HW);
    t /= HW;
    const int ch = (int)(t % (ldo / 8)), b = (int)(t / (ldo / 8));
    const int c = ch * 8 + e;
    float v = 0.0f;
    if (c < C) {
        v = g[((size_t)b * HW + pix) * ldg + goff + c];
        if (y && !(__bfloat162float(y[(((size_t)b * (ldy / 8) + (yoff + c) / 8) * HW + pix) * 8 + e]) > 0.0f)) v = 0.0f;
    }
    out[i] = __float2bfloat16_rn(v);
}

// nearest 2x upsampling of src (chunk-planar, lds channels, B x h x w) channels [0, C) into dst
// (chunk-planar, ldd channels, B x 2h x 2w) channels [doff, doff + C): one thread per 16-byte
// source pixel slot (8 channels), grid (ceil(w / 128), h, B C / 8), four 16-byte stores
__global__ void __launch_bounds__(128) k_up2(const uint4* src, int lds, int h, int w, int C, uint4* dst, int ldd,
                                             int doff) {
    grid_dependency_wait();  // launched with programmatic stream serialisation
    launch_dependents();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w) return;
    const int nch = C / 8, b = blockIdx.z / nch, ch = blockIdx.z - b * nch, W = 2 * w;
    const uint4 v = src[(((size_t)b * (lds / 8) + ch) * h + y) * w + x];
    uint4* d = dst + (((size_t)b * (ldd / 8) + doff / 8 + ch) * (2 * (size_t)h) + 2 * y) * W + 2 * x;
    d[0] = v;
    d[1] = v;
    d[W] = v;
    d[W + 1] = v;
}
// out (B, h, w, C) = sum over each 2x2 block of g (B, 2h, 2w, ldg) channels [goff, goff + C)
__global__ void k_up2_bwd(const float* g, int ldg, int goff, int B, int h, int w, int C, float* out) {
    const int i = gtid();
    if (i >= B * h * w * C) return;
    const int c = i % C, px = i / C, x = px % w, y = (px / w) % h, b = px / (w * h);
    const int W = 2 * w;
    float s = 0.0f;
#pragma unroll
    for (int d = 0; d < 4; ++d) s += g[((size_t)(b * 2 * h + 2 * y + (d >> 1)) * W + 2 * x + (d & 1)) * ldg + goff + c];
    out[i] = s;
}
// 2x2 average pooling of src (chunk-planar, lds channels, B x 2h x 2w) channels [soff, soff + C) into
// dst (chunk-planar, C channels, B x h x w): one thread per 16-byte destination pixel slot, grid
// (ceil(w / 128), h, B C / 8); each channel sums its four inputs in the order (2y, 2x), (2y, 2x+1),
// (2y+1, 2x), (2y+1, 2x+1) in fp32 and stores a quarter of the sum
__global__ void __launch_bounds__(128) k_pool2(const uint4* src, int lds, int soff, int h, int w, int C, uint4* dst) {
    grid_dependency_wait();  // launched with programmatic stream serialisation
    launch_dependents();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w) return;
    const int nch = C / 8, b = blockIdx.z / nch, ch = blockIdx.z - b * nch, W = 2 * w;
    const uint4* s0 = src + (((size_t)b * (lds / 8) + soff / 8 + ch) * (2 * (size_t)h) + 2 * y) * W + 2 * x;
    const uint4 q[4] = {s0[0], s0[1], s0[W], s0[W + 1]};
    float acc[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) acc[e] = 0.0f;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        const uint32_t wd[4] = {q[d].x, q[d].y, q[d].z, q[d].w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&wd[k]));
            acc[2 * k] += f.x;
            acc[2 * k + 1] += f.y;
        }
    }
    uint32_t o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        __nv_bfloat162 hh = __floats2bfloat162_rn(0.25f * acc[2 * k], 0.25f * acc[2 * k + 1]);
        o[k] = *reinterpret_cast<uint32_t*>(&hh);
    }
    dst[(((size_t)b * nch + ch) * h + y) * w + x] = make_uint4(o[0], o[1], o[2], o[3]);
}
// acc (B, 2h, 2w, lda) channels [aoff, aoff + C) += g (B, h, w, C) / 4 spread over each 2x2 block
__global__ void k_pool2_bwd_add(const float* g, int B, int h, int w, int C, float* acc, int lda, int aoff) {
    const int i = gtid();
    const int H = 2 * h, W = 2 * w;
    if (i >= B * H * W * C) return;
    const int c = i % C, px = i / C, X = px % W, Y = (px / W) % H, b = px / (W * H);
    acc[(size_t)px * lda + aoff + c] += 0.25f * g[((size_t)(b * h + Y / 2) * w + X / 2) * C + c];
}
// db[c] += sum over pixels of dz (chunk-planar, ld channels, B images of HW pixels) channel c: one
// block per 256-pixel chunk of one image, shared partial sums, one atomic per channel
__global__ void k_bias_grad(const bf16* dz, int ld, int B, int HW, int C, float* db) {
    __shared__ float s[256];
    for (int c = threadIdx.x; c < C; c += blockDim.x) s[c] = 0.0f;
    __syncthreads();
    const int chunks = (HW + 255) / 256;
    const int b = blockIdx.x / chunks, p0 = (blockIdx.x - b * chunks) * 256;
    for (int i = threadIdx.x; i < 256 * C; i += blockDim.x) {
        const int c = i / 256, p = p0 + (i & 255);  // consecutive threads: consecutive pixels of a channel
        if (p < HW) atomicAdd(&s[c], __bfloat162float(dz[(((size_t)b * (ld / 8) + c / 8) * HW + p) * 8 + (c & 7)]));
    }
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(&db[c], s[c]);
}
// L1 loss of pred = base + r against target (M x 3, fp32): loss_sum += sum |d|, dr[m][0..7] = scale * sign(d)
__global__ void k_l1(const float* base, const float* r, const float* target, int M, float* loss_sum, bf16* dr,
                     float scale) {
    const int m = gtid();
    float l = 0.0f;
    if (m < M) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float gsgn = 0.0f;
            if (c < 3) {
                const float d = base[(size_t)m * 3 + c] + r[(size_t)m * 3 + c] - target[(size_t)m * 3 + c];
                l += fabsf(d);
                gsgn = d > 0.0f ? scale : (d < 0.0f ? -scale : 0.0f);
            }
            dr[(size_t)m * 8 + c] = __float2bfloat16_rn(gsgn);
        }
    }
    for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss_sum, l);
}
// out = base + r (M x 3)
__global__ void k_residual(const float* base, const float* r, int n, float* out) {
    grid_dependency_wait();  // launched with programmatic stream serialisation
    launch_dependents();
    const int i = gtid();
    if (i < n) out[i] = base[i] + r[i];
}
// Adam (Kingma & Ba 2015) on fp32 master weights; wb (optional) receives the bf16 copy
__global__ void k_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2, bf16* wb) {
    const int i = gtid();
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
}
// fp32 -> bf16 copy with a row length change: dst[r][c] = c < cols ? src[r * lds + c] : 0 (c < ldd)
__global__ void k_to_bf16(const float* src, int lds, int rows, int cols, bf16* dst, int ldd) {
    const int i = gtid();
    if (i >= rows * ldd) return;
    const int r = i / ldd, c = i - r * ldd;
    dst[i] = __float2bfloat16_rn(c < cols ? src[(size_t)r * lds + c] : 0.0f);
}

// Denoiser input of one frame from the renderer's accumulation (rgb sum, count) and feature sums
// (per pixel: sum r^2, g^2, b^2, alpha, depth * alpha): x (P x 8 bf16) = (mean rgb, d / (1 + d) of
// the mean covered depth, mean alpha, per-pixel ensemble standard deviation, 0, 0); base (P x 3) =
// mean rgb.
__global__ void k_pack(const float4* accum, const float* feat, int P, bf16* x, float* base) {
    const int p = gtid();
    if (p >= P) return;
    const float4 a = accum[p];
    const float n = fmaxf(a.w, 1.0f);
    const float mr = a.x / n, mg = a.y / n, mb = a.z / n;
    float f[8] = {mr, mg, mb, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (feat) {
        const float* q = feat + (size_t)p * 8;
        const float va = fmaxf(q[0] / n - mr * mr, 0.0f) + fmaxf(q[1] / n - mg * mg, 0.0f) + fmaxf(q[2] / n - mb * mb, 0.0f);
        const float alpha = q[3] / n;
        const float depth = q[3] > 0.0f ? q[4] / q[3] : 0.0f;
        f[3] = depth / (1.0f + depth);
        f[4] = alpha;
        f[5] = sqrtf(va / 3.0f);
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) x[(size_t)p * 8 + c] = __float2bfloat16_rn(f[c]);
    base[(size_t)p * 3 + 0] = mr;
    base[(size_t)p * 3 + 1] = mg;
    base[(size_t)p * 3 + 2] = mb;
}

// Training batch: crop b takes the ch x cw window at (y0, x0) of image img from the stacked frames
// (x: N x H x W x 8 bf16, base and target: N x H x W x 3 fp32); crops[b] = (img, y0, x0). A window
// outside the frames gives zeros and sets bit 16 of *err.
__global__ void k_crop(const bf16* x, const float* base, const float* target, int N, int H, int W, const int* crops,
                       int B, int ch, int cw, bf16* xb, float* baseb, float* targetb, uint32_t* err) {
    const int i = gtid();
    if (i >= B * ch * cw) return;
    const int b = i / (ch * cw), yx = i - b * ch * cw, y = yx / cw, xq = yx - y * cw;
    const int img = crops[3 * b], y0 = crops[3 * b + 1], x0 = crops[3 * b + 2];
    if (img < 0 || img >= N || y0 < 0 || y0 + ch > H || x0 < 0 || x0 + cw > W) {
        *reinterpret_cast<uint4*>(xb + (size_t)i * 8) = make_uint4(0u, 0u, 0u, 0u);
        for (int c = 0; c < 3; ++c) baseb[(size_t)i * 3 + c] = targetb[(size_t)i * 3 + c] = 0.0f;
        if (yx == 0 && err) atomicOr(err, 1u << 16);
        return;
    }
    const size_t src = ((size_t)img * H + y0 + y) * W + x0 + xq;
    *reinterpret_cast<uint4*>(xb + (size_t)i * 8) = *reinterpret_cast<const uint4*>(x + src * 8);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        baseb[(size_t)i * 3 + c] = base[src * 3 + c];
        targetb[(size_t)i * 3 + c] = target[src * 3 + c];
    }
}
// *sum += sum over M pixels of channel c of the bf16 tensor x (M x ld): one partial per warp
__global__ void k_channel_sum(const bf16* x, int ld, int c, int M, float* sum) {
    float s = 0.0f;
    for (int m = gtid(); m < M; m += gridDim.x * blockDim.x) s += __bfloat162float(x[(size_t)m * ld + c]);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s != 0.0f) atomicAdd(sum, s);
}
// rgb (P x 3) = accumulated colour / max(count, 1) of the renderer's accumulation (P float4)
__global__ void k_mean_rgb(const float4* accum, int P, float* rgb) {
    const int p = gtid();
    if (p >= P) return;
    const float4 a = accum[p];
    const float n = fmaxf(a.w, 1.0f);
    rgb[(size_t)p * 3 + 0] = a.x / n;
    rgb[(size_t)p * 3 + 1] = a.y / n;
    rgb[(size_t)p * 3 + 2] = a.z / n;
}
}  // namespace dn
}  // namespace gpsb

using namespace gpsb;
using namespace gpsb::dn;

template <int BN>
static cudaError_t launch_fwd(const ConvFwd& p, cudaStream_t st) {
    ConvFwdN<BN> q;
    static_cast<ConvFwd&>(q) = p;
    const size_t smem = umma::smem_bytes_async<BN, fwd_stages<BN>()>();
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

static inline int grid_of(long n) { return (int)((n + 255) / 256); }

int gpsb_dn_relu_bwd(const float* g, int ldg, int goff, const void* y, int ldy, int yoff, int B, int HW, int C,
                     void* out, int ldo, void* stream) {
    if (C > ldo || ldo % 8 || ldy % 8 || yoff % 8) return (int)cudaErrorInvalidValue;
    k_relu_bwd<<<grid_of((long)B * HW * ldo), 256, 0, (cudaStream_t)stream>>>(g, ldg, goff, (const bf16*)y, ldy, yoff,
                                                                               B, HW, C, (bf16*)out, ldo);
    return (int)cudaGetLastError();
}
int gpsb_dn_up2(const void* src, int lds, int B, int h, int w, int C, void* dst, int ldd, int doff, void* stream) {
    if (C % 8 || lds % 8 || ldd % 8 || doff % 8 || B < 1 || h < 1 || w < 1 || h > 65535 || (long)B * (C / 8) > 65535 ||
        ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15u))
        return (int)cudaErrorInvalidValue;
    return (int)launch_pdl(k_up2, dim3((w + 127) / 128, h, B * (C / 8)), dim3(128), 0, (cudaStream_t)stream,
                           (const uint4*)src, lds, h, w, C, (uint4*)dst, ldd, doff);
}
int gpsb_dn_up2_bwd(const float* g, int ldg, int goff, int B, int h, int w, int C, float* out, void* stream) {
    k_up2_bwd<<<grid_of((long)B * h * w * C), 256, 0, (cudaStream_t)stream>>>(g, ldg, goff, B, h, w, C, out);
    return (int)cudaGetLastError();
}
int gpsb_dn_pool2(const void* src, int lds, int soff, int B, int h, int w, int C, void* dst, void* stream) {
    if (C % 8 || lds % 8 || soff % 8 || B < 1 || h < 1 || w < 1 || h > 65535 || (long)B * (C / 8) > 65535 ||
        ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15u))
        return (int)cudaErrorInvalidValue;
    return (int)launch_pdl(k_pool2, dim3((w + 127) / 128, h, B * (C / 8)), dim3(128), 0, (cudaStream_t)stream,
                           (const uint4*)src, lds, soff, h, w, C, (uint4*)dst);
}
int gpsb_dn_pool2_bwd_add(const float* g, int B, int h, int w, int C, float* acc, int lda, int aoff, void* stream) {
    k_pool2_bwd_add<<<grid_of(4L * B * h * w * C), 256, 0, (cudaStream_t)stream>>>(g, B, h, w, C, acc, lda, aoff);
    return (int)cudaGetLastError();
}
int gpsb_dn_bias_grad(const void* dz, int ld, int B, int HW, int C, float* db, void* stream) {
    if (C > 256 || ld % 8 || C > ld) return (int)cudaErrorInvalidValue;
    k_bias_grad<<<B * ((HW + 255) / 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)dz, ld, B, HW, C, db);
    return (int)cudaGetLastError();
}
int gpsb_dn_l1(const float* base, const float* r, const float* target, int M, float* loss_sum, void* dr, float scale,
               void* stream) {
    k_l1<<<grid_of(M), 256, 0, (cudaStream_t)stream>>>(base, r, target, M, loss_sum, (bf16*)dr, scale);
    return (int)cudaGetLastError();
}
int gpsb_dn_residual(const float* base, const float* r, int n, float* out, void* stream) {
    if (n <= 0) return (int)cudaSuccess;
    const cudaError_t e = launch_pdl(k_residual, dim3(grid_of(n)), dim3(256), 0, (cudaStream_t)stream, base, r, n, out);
    if (e != cudaSuccess) return (int)e;
    return (int)cudaGetLastError();
}
int gpsb_dn_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps, int t,
                 void* wb, void* stream) {
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    k_adam<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2, (bf16*)wb);
    return (int)cudaGetLastError();
}
int gpsb_dn_to_bf16(const float* src, int lds, int rows, int cols, void* dst, int ldd, void* stream) {
    k_to_bf16<<<grid_of((long)rows * ldd), 256, 0, (cudaStream_t)stream>>>(src, lds, rows, cols, (bf16*)dst, ldd);
    return (int)cudaGetLastError();
}
int gpsb_dn_pack(const void* accum, const float* feat, int P, void* x, float* base, void* stream) {
    k_pack<<<grid_of(P), 256, 0, (cudaStream_t)stream>>>((const float4*)accum, feat, P, (bf16*)x, base);
    return (int)cudaGetLastError();
}
int gpsb_dn_channel_sum(const void* x, int ld, int c, int M, float* sum, void* stream) {
    if (c < 0 || c >= ld || M < 0) return (int)cudaErrorInvalidValue;
    const int blocks = grid_of(M) < 1184 ? grid_of(M) : 1184;
    if (blocks > 0) k_channel_sum<<<blocks, 256, 0, (cudaStream_t)stream>>>((const bf16*)x, ld, c, M, sum);
    return (int)cudaGetLastError();
}
int gpsb_dn_mean_rgb(const void* accum, int P, float* rgb, void* stream) {
    if (P > 0) k_mean_rgb<<<grid_of(P), 256, 0, (cudaStream_t)stream>>>((const float4*)accum, P, rgb);
    return (int)cudaGetLastError();
}
int gpsb_dn_crop(const void* x, const float* base, const float* target, int N, int H, int W, const int* crops, int B,
                 int ch, int cw, void* xb, float* baseb, float* targetb, void* stream, uint32_t* err) {
    k_crop<<<grid_of((long)B * ch * cw), 256, 0, (cudaStream_t)stream>>>((const bf16*)x, base, target, N, H, W, crops, B,
                                                                          ch, cw, (bf16*)xb, baseb, targetb, err);
    return (int)cudaGetLastError();
}

}  // extern "C"
