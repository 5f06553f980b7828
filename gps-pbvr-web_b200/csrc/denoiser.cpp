// The learned denoiser behind the C ABI: a 3-level U-Net (3x3 convolutions of 32/64/128 channels,
// ReLU, 2x2 average pooling, nearest upsampling with skip concatenation, a final convolution to a
// residual added to the few-ensemble mean colour) run on the library's kernels (conv3 on the tensor
// cores, the element-wise steps of denoise.cu), and the denoised frame of a renderer: a few
// ensembles with per-pixel feature sums, the per-frame variance check, the network, or the plain
// accumulation of more ensembles when the check fails. The reference has no denoiser; this is the
// host sequencing a Rust caller binds next to gpsb_render_ensembles, with no PyTorch involved.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <string>
#include <vector>

#include "gpsb200.h"
#include "internal.h"

namespace gpsb {
cudaStream_t renderer_stream(gpsb_renderer* r);
int renderer_device(gpsb_renderer* r);
}

namespace {

struct Layer {
    const char* name;
    int cin, cin_real, cout;
};
// (name, padded input channels, real input channels, output channels); ReLU after all but c6
const Layer kLayers[GPSB_DN_LAYERS] = {
    {"c1a", 8, 6, 32},    {"c1b", 32, 32, 32},    {"c2a", 32, 32, 64},    {"c2b", 64, 64, 64},
    {"c3a", 64, 64, 128}, {"c3b", 128, 128, 128}, {"c4a", 192, 192, 64}, {"c4b", 64, 64, 64},
    {"c5a", 96, 96, 32},  {"c5b", 32, 32, 32},    {"c6", 32, 32, 3}};

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t n) {
        if (p && n <= bytes) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, n < 256 ? 256 : n);
        if (e == cudaSuccess) bytes = n < 256 ? 256 : n;
        else p = nullptr;
        return e;
    }
    template <class T> T* as() const { return (T*)p; }
};

}  // namespace

struct gpsb_denoiser {
    int device = 0;
    float gate_limit = 0.0f;
    bool loaded[GPSB_DN_LAYERS] = {};
    Buf wt[GPSB_DN_LAYERS], bias[GPSB_DN_LAYERS];
    // activations of the current frame size (batch 1)
    uint32_t W = 0, H = 0;
    Buf x, base, feat, a1, cat1, p1, a2, cat2, p2, a3, b3, d2a, d2, d1a, d1, r, pred, err, sum;
    // the U-Net's 16 launches captured once per frame size and replayed as one graph launch (the
    // kernels' arguments, tensor maps included, are fixed for fixed buffers)
    cudaStream_t capture = nullptr;
    cudaGraphExec_t graph = nullptr;
    uint32_t graph_w = 0, graph_h = 0;
    bool graph_unavailable = false;  // a capture failed: keep launching directly
    std::string error;
};

static void drop_graph(gpsb_denoiser* d) {
    if (d->graph) cudaGraphExecDestroy(d->graph);
    d->graph = nullptr;
    d->graph_w = d->graph_h = 0;
}

static gpsb_status dn_fail(gpsb_denoiser* d, gpsb_status s, const std::string& msg) {
    if (d) d->error = msg;
    return s;
}

#define DCK(d, call, what)                                                                              \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return dn_fail(d, e_ == cudaErrorMemoryAllocation ? GPSB_ERR_OUT_OF_MEMORY : GPSB_ERR_CUDA, \
                           std::string(what) + ": " + cudaGetErrorString(e_));                         \
    } while (0)
#define DK(d, call, what) DCK(d, (cudaError_t)(call), what)

extern "C" {

gpsb_status gpsb_denoiser_create(int device, gpsb_denoiser** out) {
    if (!out) return GPSB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return GPSB_ERR_CUDA;
    gpsb_denoiser* d = new gpsb_denoiser();
    d->device = device;
    *out = d;
    return GPSB_OK;
}

void gpsb_denoiser_destroy(gpsb_denoiser* d) {
    if (!d) return;
    cudaSetDevice(d->device);
    drop_graph(d);
    if (d->capture) cudaStreamDestroy(d->capture);
    for (int l = 0; l < GPSB_DN_LAYERS; ++l) {
        d->wt[l].release();
        d->bias[l].release();
    }
    for (Buf* b : {&d->x, &d->base, &d->feat, &d->a1, &d->cat1, &d->p1, &d->a2, &d->cat2, &d->p2, &d->a3, &d->b3,
                   &d->d2a, &d->d2, &d->d1a, &d->d1, &d->r, &d->pred, &d->err, &d->sum})
        b->release();
    delete d;
}

const char* gpsb_denoiser_last_error(const gpsb_denoiser* d) { return d ? d->error.c_str() : ""; }

int gpsb_denoiser_graph_state(const gpsb_denoiser* d) {
    if (!d) return 0;
    if (d->graph_unavailable) return -1;
    return (d->graph && d->graph_w == d->W && d->graph_h == d->H) ? 1 : 0;
}

gpsb_status gpsb_denoiser_layer_shape(uint32_t layer, uint32_t* cin, uint32_t* cin_real, uint32_t* cout) {
    if (layer >= GPSB_DN_LAYERS) return GPSB_ERR_INVALID_ARGUMENT;
    if (cin) *cin = (uint32_t)kLayers[layer].cin;
    if (cin_real) *cin_real = (uint32_t)kLayers[layer].cin_real;
    if (cout) *cout = (uint32_t)kLayers[layer].cout;
    return GPSB_OK;
}

gpsb_status gpsb_denoiser_set_layer(gpsb_denoiser* d, uint32_t layer, const float* w, const float* b) {
    if (!d || !w || !b || layer >= GPSB_DN_LAYERS) return dn_fail(d, GPSB_ERR_INVALID_ARGUMENT, "bad layer or null");
    const Layer& L = kLayers[layer];
    cudaSetDevice(d->device);
    drop_graph(d);
    const int K = 9 * L.cin, kp = (K + 63) / 64 * 64;
    // fp32 rows [cout][kp] on the device, then bf16, then the conv3 arrangement
    Buf wf, wb;
    DCK(d, wf.ensure((size_t)L.cout * kp * 4), "weights");
    DCK(d, wb.ensure((size_t)L.cout * kp * 2), "weights");
    std::vector<float> rows((size_t)L.cout * kp, 0.0f);
    for (int n = 0; n < L.cout; ++n) memcpy(&rows[(size_t)n * kp], w + (size_t)n * K, (size_t)K * 4);
    cudaError_t e = cudaMemcpy(wf.p, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = (cudaError_t)gpsb_dn_to_bf16(wf.as<float>(), kp, L.cout, kp, wb.p, kp, nullptr);
    const size_t tb = (size_t)gpsb_dn_conv3_weight_bytes(L.cout, L.cin);
    if (e == cudaSuccess) e = d->wt[layer].ensure(tb);
    if (e == cudaSuccess) e = (cudaError_t)gpsb_dn_conv3_weights(wb.p, L.cout, L.cin, kp, d->wt[layer].p, nullptr);
    if (e == cudaSuccess) e = d->bias[layer].ensure((size_t)L.cout * 4);
    if (e == cudaSuccess) e = cudaMemcpy(d->bias[layer].p, b, (size_t)L.cout * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    wf.release();
    wb.release();
    DCK(d, e, "set layer");
    d->loaded[layer] = true;
    return GPSB_OK;
}

gpsb_status gpsb_denoiser_set_gate(gpsb_denoiser* d, float gate_limit) {
    if (!d) return GPSB_ERR_INVALID_ARGUMENT;
    d->gate_limit = gate_limit;
    return GPSB_OK;
}

}  // extern "C"

static gpsb_status ensure_frame(gpsb_denoiser* d, uint32_t W, uint32_t H) {
    if (d->W == W && d->H == H && d->x.p) return GPSB_OK;
    drop_graph(d);
    const size_t P = (size_t)W * H, P2 = P / 4, P4 = P / 16;
    const size_t bf = 2;
    struct {
        Buf* b;
        size_t bytes;
    } plan[] = {{&d->x, P * 8 * bf},     {&d->base, P * 3 * 4},   {&d->feat, P * 8 * 4},   {&d->a1, P * 32 * bf},
                {&d->cat1, P * 96 * bf}, {&d->p1, P2 * 32 * bf},  {&d->a2, P2 * 64 * bf},  {&d->cat2, P2 * 192 * bf},
                {&d->p2, P4 * 64 * bf},  {&d->a3, P4 * 128 * bf}, {&d->b3, P4 * 128 * bf}, {&d->d2a, P2 * 64 * bf},
                {&d->d2, P2 * 64 * bf},  {&d->d1a, P * 32 * bf},  {&d->d1, P * 32 * bf},   {&d->r, P * 3 * 4},
                {&d->pred, P * 3 * 4},   {&d->err, 16},           {&d->sum, 16}};
    for (auto& q : plan) {
        q.b->release();
        DCK(d, q.b->ensure(q.bytes), "denoiser buffers");
    }
    d->W = W;
    d->H = H;
    return GPSB_OK;
}

// The U-Net on d->x / d->base into d->pred (all enqueued on st).
static gpsb_status unet(gpsb_denoiser* d, cudaStream_t st) {
    const int H = (int)d->H, W = (int)d->W, h2 = H / 2, w2 = W / 2, h4 = H / 4, w4 = W / 4;
    uint32_t* err = d->err.as<uint32_t>();
    auto conv = [&](int l, const Buf& x, int ldx, int h, int w, Buf& out, int ldo, int ooff, bool f32, bool relu) {
        const Layer& L = kLayers[l];
        return gpsb_dn_conv3(x.p, ldx, 0, L.cin, 1, h, w, d->wt[l].p, L.cout, d->bias[l].as<float>(), out.p, ldo, ooff,
                             f32 ? 1 : 0, relu ? 1 : 0, st, err);
    };
    DK(d, conv(0, d->x, 8, H, W, d->a1, 32, 0, false, true), "c1a");
    DK(d, conv(1, d->a1, 32, H, W, d->cat1, 96, 64, false, true), "c1b");
    DK(d, gpsb_dn_pool2(d->cat1.p, 96, 64, 1, h2, w2, 32, d->p1.p, st), "pool");
    DK(d, conv(2, d->p1, 32, h2, w2, d->a2, 64, 0, false, true), "c2a");
    DK(d, conv(3, d->a2, 64, h2, w2, d->cat2, 192, 128, false, true), "c2b");
    DK(d, gpsb_dn_pool2(d->cat2.p, 192, 128, 1, h4, w4, 64, d->p2.p, st), "pool");
    DK(d, conv(4, d->p2, 64, h4, w4, d->a3, 128, 0, false, true), "c3a");
    DK(d, conv(5, d->a3, 128, h4, w4, d->b3, 128, 0, false, true), "c3b");
    DK(d, gpsb_dn_up2(d->b3.p, 128, 1, h4, w4, 128, d->cat2.p, 192, 0, st), "up");
    DK(d, conv(6, d->cat2, 192, h2, w2, d->d2a, 64, 0, false, true), "c4a");
    DK(d, conv(7, d->d2a, 64, h2, w2, d->d2, 64, 0, false, true), "c4b");
    DK(d, gpsb_dn_up2(d->d2.p, 64, 1, h2, w2, 64, d->cat1.p, 96, 0, st), "up");
    DK(d, conv(8, d->cat1, 96, H, W, d->d1a, 32, 0, false, true), "c5a");
    DK(d, conv(9, d->d1a, 32, H, W, d->d1, 32, 0, false, true), "c5b");
    DK(d, conv(10, d->d1, 32, H, W, d->r, 3, 0, true, false), "c6");
    DK(d, gpsb_dn_residual(d->base.as<float>(), d->r.as<float>(), H * W * 3, d->pred.as<float>(), st), "residual");
    return GPSB_OK;
}

// The U-Net on st: the captured graph of this frame size, or (first frame of a size) the direct
// launches followed by one capture of the same launches on the denoiser's own stream.
static gpsb_status run_unet(gpsb_denoiser* d, cudaStream_t st) {
    if (d->graph && d->graph_w == d->W && d->graph_h == d->H) {
        DCK(d, cudaGraphLaunch(d->graph, st), "graph launch");
        return GPSB_OK;
    }
    gpsb_status s = unet(d, st);
    if (s != GPSB_OK || d->graph_unavailable) return s;
    if (!d->capture && cudaStreamCreateWithFlags(&d->capture, cudaStreamNonBlocking) != cudaSuccess) {
        d->capture = nullptr;
        d->graph_unavailable = true;
        cudaGetLastError();
        return GPSB_OK;
    }
    cudaGraph_t g = nullptr;
    bool ok = cudaStreamBeginCapture(d->capture, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        const std::string keep = d->error;
        const bool launched = unet(d, d->capture) == GPSB_OK;
        d->error = keep;
        ok = cudaStreamEndCapture(d->capture, &g) == cudaSuccess && launched && g &&
             cudaGraphInstantiate(&d->graph, g, 0) == cudaSuccess;
    }
    if (g) cudaGraphDestroy(g);
    if (ok) {
        d->graph_w = d->W;
        d->graph_h = d->H;
    } else {
        d->graph = nullptr;
        d->graph_unavailable = true;
        cudaGetLastError();
    }
    return GPSB_OK;
}

static gpsb_status check_loaded(gpsb_denoiser* d) {
    for (int l = 0; l < GPSB_DN_LAYERS; ++l)
        if (!d->loaded[l]) return dn_fail(d, GPSB_ERR_STATE, std::string("layer ") + kLayers[l].name + " not set");
    return GPSB_OK;
}

extern "C" {

gpsb_status gpsb_denoiser_forward(gpsb_denoiser* d, const void* x_dev, const float* base_dev, uint32_t width,
                                  uint32_t height, float* pred_dev, void* cuda_stream) {
    if (!d || !x_dev || !base_dev || !pred_dev) return dn_fail(d, GPSB_ERR_INVALID_ARGUMENT, "null argument");
    if (width == 0 || height == 0 || width % 4 || height % 4)
        return dn_fail(d, GPSB_ERR_INVALID_ARGUMENT, "width and height must be positive multiples of 4");
    gpsb_status s = check_loaded(d);
    if (s != GPSB_OK) return s;
    cudaSetDevice(d->device);
    s = ensure_frame(d, width, height);
    if (s != GPSB_OK) return s;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const size_t P = (size_t)width * height;
    DCK(d, cudaMemcpyAsync(d->x.p, x_dev, P * 16, cudaMemcpyDeviceToDevice, st), "input");
    DCK(d, cudaMemcpyAsync(d->base.p, base_dev, P * 12, cudaMemcpyDeviceToDevice, st), "input");
    DCK(d, cudaMemsetAsync(d->err.p, 0, 4, st), "error word");
    s = run_unet(d, st);
    if (s != GPSB_OK) return s;
    DCK(d, cudaMemcpyAsync(pred_dev, d->pred.p, P * 12, cudaMemcpyDeviceToDevice, st), "output");
    uint32_t e = 0;
    DCK(d, cudaMemcpyAsync(&e, d->err.p, 4, cudaMemcpyDeviceToHost, st), "error word");
    DCK(d, cudaStreamSynchronize(st), "synchronise");
    if (e) return dn_fail(d, GPSB_ERR_TIMEOUT, "a bounded device-side wait of the network gave up");
    return GPSB_OK;
}

gpsb_status gpsb_render_denoised(gpsb_renderer* r, gpsb_denoiser* d, const gpsb_camera* cam, const gpsb_params* p,
                                 uint32_t first_seed, uint32_t ensembles, float gate_limit,
                                 uint32_t fallback_ensembles, float* rgb_host, int* used_denoiser, float* check) {
    if (!r || !d || !cam || !p || !rgb_host) return dn_fail(d, GPSB_ERR_INVALID_ARGUMENT, "null argument");
    if (ensembles == 0) return dn_fail(d, GPSB_ERR_INVALID_ARGUMENT, "at least one ensemble");
    uint32_t W = 0, H = 0, side = 0;
    gpsb_size(r, &W, &H, &side);
    if (W == 0 || H == 0 || W % 4 || H % 4)
        return dn_fail(d, GPSB_ERR_INVALID_ARGUMENT, "the denoiser needs width and height divisible by 4");
    gpsb_status s = check_loaded(d);
    if (s != GPSB_OK) return s;
    if (gpsb::renderer_device(r) != d->device) return dn_fail(d, GPSB_ERR_INVALID_ARGUMENT, "renderer on another device");
    cudaSetDevice(d->device);
    s = ensure_frame(d, W, H);
    if (s != GPSB_OK) return s;
    cudaStream_t st = gpsb::renderer_stream(r);
    const size_t P = (size_t)W * H;
    const float limit = gate_limit > 0.0f ? gate_limit : d->gate_limit;
    // few ensembles with the per-pixel feature sums (colour squares, coverage, covered depth)
    DCK(d, cudaMemsetAsync(d->feat.p, 0, P * 32, st), "features");
    s = gpsb_reset_accum(r);
    if (s == GPSB_OK) s = gpsb_set_feature_accum(r, d->feat.as<float>());
    if (s == GPSB_OK) s = gpsb_render_ensembles(r, cam, p, first_seed, ensembles);
    gpsb_set_feature_accum(r, nullptr);
    if (s != GPSB_OK) return dn_fail(d, s, gpsb_last_error(r));
    void* acc = nullptr;
    gpsb_accum_device_ptr(r, &acc);
    DK(d, gpsb_dn_pack(acc, d->feat.as<float>(), (int)P, d->x.p, d->base.as<float>(), st), "pack");
    // the per-frame variance check: mean per-pixel ensemble standard deviation (feature 5)
    DCK(d, cudaMemsetAsync(d->sum.p, 0, 4, st), "check");
    DK(d, gpsb_dn_channel_sum(d->x.p, 8, 5, (int)P, d->sum.as<float>(), st), "check");
    float sum = 0.0f;
    DCK(d, cudaMemcpyAsync(&sum, d->sum.p, 4, cudaMemcpyDeviceToHost, st), "check");
    DCK(d, cudaStreamSynchronize(st), "synchronise");
    const float mean_sd = sum / (float)P;
    if (check) *check = mean_sd;
    const bool use = mean_sd <= limit;
    if (used_denoiser) *used_denoiser = use ? 1 : 0;
    if (use) {
        DCK(d, cudaMemsetAsync(d->err.p, 0, 4, st), "error word");
        s = run_unet(d, st);
        if (s != GPSB_OK) return s;
        DCK(d, cudaMemcpyAsync(rgb_host, d->pred.p, P * 12, cudaMemcpyDeviceToHost, st), "read frame");
        uint32_t e = 0;
        DCK(d, cudaMemcpyAsync(&e, d->err.p, 4, cudaMemcpyDeviceToHost, st), "error word");
        DCK(d, cudaStreamSynchronize(st), "synchronise");
        if (e) return dn_fail(d, GPSB_ERR_TIMEOUT, "a bounded device-side wait of the network gave up");
        return GPSB_OK;
    }
    // outside what the network was trained on: the plain accumulation of fallback_ensembles
    if (fallback_ensembles > ensembles) {
        s = gpsb_render_ensembles(r, cam, p, first_seed + ensembles, fallback_ensembles - ensembles);
        if (s != GPSB_OK) return dn_fail(d, s, gpsb_last_error(r));
    }
    DK(d, gpsb_dn_mean_rgb(acc, (int)P, d->pred.as<float>(), st), "mean colour");
    DCK(d, cudaMemcpyAsync(rgb_host, d->pred.p, P * 12, cudaMemcpyDeviceToHost, st), "read frame");
    DCK(d, cudaStreamSynchronize(st), "synchronise");
    return GPSB_OK;
}

}  // extern "C"
