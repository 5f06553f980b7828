// GPU-side decode of a binary little-endian 3DGS PLY (next step before the hot path): the header
// is parsed on the host exactly as gpsb_load_ply does (crates/gps-io/src/lib.rs:165-238), the
// vertex block is copied to the device once, and one thread per vertex reads its properties by
// offset and type, applies the activation (gps-io lib.rs:84-96) and GpuGaussian::from_activated
// (gps.rs:41-49) in the host loader's arithmetic (double, no contraction), and writes the 64-byte
// splat and the channel-major SH rest. The first non-finite value (in vertex order, then
// property order) is reported with the host loader's message.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include <string>

#include "ply_layout.h"

namespace gpsb {
namespace {

struct PlyDev {
    uint32_t off[59];
    uint8_t type[59];
    uint32_t nprop, stride, per_ch;
};

__device__ __forceinline__ double read_prop(const uint8_t* b, uint8_t t) {
    switch (t) {
        case 0: return (double)(int8_t)b[0];
        case 1: return (double)b[0];
        case 2: return (double)(int16_t)(b[0] | (b[1] << 8));
        case 3: return (double)(uint16_t)(b[0] | (b[1] << 8));
        case 4: case 5: case 6: {
            uint32_t u = (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
            if (t == 4) return (double)(int32_t)u;
            if (t == 5) return (double)u;
            return (double)__uint_as_float(u);
        }
        default: {
            uint64_t u = 0;
            for (int i = 7; i >= 0; --i) u = (u << 8) | b[i];
            return __longlong_as_double((long long)u);
        }
    }
}

__global__ void k_ply_decode(const uint8_t* __restrict__ body, size_t n, PlyDev L, float4* splats, float* sh,
                             unsigned long long* first_bad) {
    const size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const uint8_t* rec = body + v * L.stride;
    float f[14];
    bool bad = false;
    uint32_t bad_field = 0;
    for (int k = 0; k < 14; ++k) {
        f[k] = (float)read_prop(rec + L.off[k], L.type[k]);  // (double)(float) of the host loader
        if (!bad && !isfinite(f[k])) { bad = true; bad_field = (uint32_t)k; }
    }
    for (uint32_t r = 14; r < L.nprop; ++r) {
        const float x = (float)read_prop(rec + L.off[r], L.type[r]);
        if (!bad && !isfinite(x)) { bad = true; bad_field = 14; }
        if (sh) sh[v * 3 * L.per_ch + (r - 14)] = x;
    }
    if (bad) {
        atomicMin(first_bad, ((unsigned long long)v << 8) | bad_field);
        return;
    }
    const double op = 1.0 / (1.0 + exp(-(double)f[6]));
    const double c0 = 0.28209479177387814;
    float4* g = splats + v * 4;
    g[0] = make_float4(f[0], f[1], f[2], (float)op);
    g[1] = make_float4(f[7], f[8], f[9], 0.0f);
    g[2] = make_float4(f[10], f[11], f[12], f[13]);
    g[3] = make_float4((float)((double)f[3] * c0 + 0.5), (float)((double)f[4] * c0 + 0.5), (float)((double)f[5] * c0 + 0.5),
                       0.0f);
}

}  // namespace
}  // namespace gpsb

using namespace gpsb;

extern "C" gpsb_status gpsb_load_ply_device(const uint8_t* bytes, size_t len, size_t* n_out, uint32_t* sh_degree_out,
                                            gpsb_gaussian* splats_dev, float* sh_rest_dev, void* cuda_stream) {
    if (!bytes || !n_out || !sh_degree_out) return GPSB_ERR_INVALID_ARGUMENT;
    PlyLayout h;
    gpsb_status s = ply_layout(bytes, len, &h);
    if (s != GPSB_OK) return s;
    if (!h.binary) return ply_error("GPU decode needs binary_little_endian vertex data (use gpsb_load_ply for ASCII)");
    *n_out = h.count;
    *sh_degree_out = h.degree;
    if (!splats_dev || h.count == 0) return GPSB_OK;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    PlyDev L;
    for (uint32_t i = 0; i < h.nprop; ++i) {
        L.off[i] = h.off[i];
        L.type[i] = h.type[i];
    }
    L.nprop = h.nprop;
    L.stride = (uint32_t)h.stride;
    L.per_ch = h.degree ? (h.degree + 1) * (h.degree + 1) - 1 : 0;
    const size_t body_bytes = h.count * h.stride;
    uint8_t* body = nullptr;
    unsigned long long* bad = nullptr;
    cudaError_t e = cudaMalloc(&body, body_bytes + 16);
    if (e == cudaSuccess) e = cudaMalloc(&bad, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0xFF, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(body, bytes + h.data_start, body_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_ply_decode<<<(unsigned)((h.count + 255) / 256), 256, 0, st>>>(body, h.count, L, (float4*)splats_dev,
                                                                           h.degree ? sh_rest_dev : nullptr, bad);
        e = cudaGetLastError();
    }
    unsigned long long first = ~0ull;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&first, bad, sizeof first, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (body) cudaFree(body);
    if (bad) cudaFree(bad);
    if (e != cudaSuccess) {
        ply_error((std::string("CUDA error in PLY decode: ") + cudaGetErrorString(e)).c_str());
        return GPSB_ERR_CUDA;
    }
    if (first != ~0ull) {
        static const char* field_of[15] = {"position", "position", "position", "f_dc", "f_dc", "f_dc", "opacity", "scale",
                                           "scale", "scale", "rot", "rot", "rot", "rot", "f_rest"};
        const unsigned long long v = first >> 8;
        const unsigned field = (unsigned)(first & 0xFF);
        return ply_error((std::string("non-finite value in '") + field_of[field < 15 ? field : 14] + "' at vertex " +
                          std::to_string(v)).c_str());
    }
    return GPSB_OK;
}
